"""Benchmark of the B200 micromagnetic step (one JSON line on rank 0).

Workload (default): the large 3D precision configuration — a film of 512 x 512 x 16 cells
of 2 x 2 x 2 nm (padded FFT 1024 x 1024 x 32), Ms = 1.1e6 A/m, A = 1.5e-11 J/m, uniaxial
K1 = 5e5 J/m^3 along z, interfacial DMI D = 1.5e-3 J/m^2, alpha = 0.1, initial m = +z with
seeded 0..15 degree tilts, RKDP54 with relative error tolerance 1e-5, mixed precision
(FP32 FFTs and stages, FP64 tensor build and error norm). A step is one accepted RKDP54
step (six field evaluations). Data is synthetic (seeded), built here.

  value      Mcell-steps/s over the timed steps, state resident in HBM (device-event time,
             max over ranks, aggregate over ranks)
  e2e        the same metric through the C ABI with host buffers: set M from pinned host
             memory, run, read M back, all inside the timed region
  roofline   the dominant kernel's algorithmic bytes per launch / its average launch time
  cpu_baseline  the reference's own CPU demag convolution (compiled from its sources,
             oracle/_ref) on a bounded sample: 256 x 256 x 16 cells of the same film,
             6 H_demag evaluations per step

--impl reference runs that CPU reference arm alone with the same metric and config.
Multi-GPU: independent replicas, one per rank (the path has no data exchange).
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

def batch_systems(nsys=256, seed=3):
    """The batching workload: independent films with Nx, Ny drawn log-uniformly from
    {64, 96, 128, 192, 256, 384, 512} (uniform over that log-spaced set), Nz from {1, 2, 4},
    4 x 4 x 3 nm cells, Ms ~ U[4e5, 1.4e6], A ~ U[0.8e-11, 2e-11], alpha ~ U[0.01, 0.5] (seeded)."""
    rng = np.random.default_rng(seed)
    sizes = [64, 96, 128, 192, 256, 384, 512]
    out = []
    for q in range(nsys):
        n = (int(rng.choice(sizes)), int(rng.choice(sizes)), int(rng.choice([1, 2, 4])))
        out.append(dict(n=n, h=(4e-9, 4e-9, 3e-9), o=(0.0, 0.0, 0.0), Ms=float(rng.uniform(4e5, 1.4e6)), K1=0.0,
                        A=float(rng.uniform(0.8e-11, 2e-11)), alpha=float(rng.uniform(0.01, 0.5)), modules=1 | 2))
    return out


CONFIGS = {
    "film3d_512x512x16": dict(n=(512, 512, 16), h=(2e-9, 2e-9, 2e-9), Ms=1.1e6, A=1.5e-11, K1=5e5, D=1.5e-3,
                              alpha=0.1, modules=1 | 4 | 8 | 16, eval="RKDP54", dt=1e-14, tol=1e-5, init="tilt"),
    # the same film under RK4 with the demag field extrapolated quadratically between steps
    "film3d_512x512x16_rk4_es3": dict(n=(512, 512, 16), h=(2e-9, 2e-9, 2e-9), Ms=1.1e6, A=1.5e-11, K1=5e5,
                                      D=1.5e-3, alpha=0.1, modules=1 | 4 | 8 | 16, eval="RK4", dt=1e-14,
                                      tol=1e-5, init="tilt", evalspeedup=3),
    # the same film at half thickness: the small case for full ncu captures of the stage kernel
    "film3d_512x512x8": dict(n=(512, 512, 8), h=(2e-9, 2e-9, 2e-9), Ms=1.1e6, A=1.5e-11, K1=5e5, D=1.5e-3,
                             alpha=0.1, modules=1 | 4 | 8 | 16, eval="RKDP54", dt=1e-14, tol=1e-5, init="tilt"),
    "film2d_128x64": dict(n=(128, 64, 1), h=(5e-9, 5e-9, 3e-9), Ms=8e5, A=1.3e-11, K1=0.0, D=0.0, alpha=0.5,
                          grel=2.211e5 / 2.212761569e5, modules=1 | 2 | 16, Ha=(1e3, 0, 0), eval="RK4", dt=1e-13,
                          init="sphere"),
    "film2d_256x256": dict(n=(256, 256, 1), h=(4e-9, 4e-9, 3e-9), Ms=8e5, A=1.3e-11, K1=1e5, D=0.0, alpha=0.02,
                           modules=1 | 2 | 8 | 16, Ha=(0, 0, 0), eval="RK4", dt=1e-13, init="sphere"),
    # three stacked meshes with different cellsizes, 1 nm spacers, one multilayered convolution
    # (3D common grid n = (1024, 1024, 2), FFT 2048 x 2048 x 4)
    "multilayer_stack3": dict(meshes=[dict(n=(1024, 1024, 1), h=(2e-9, 2e-9, 1e-9), o=(0, 0, 0), Ms=1.4e6, K1=0.0,
                                           modules=1 | 2),
                                      dict(n=(512, 512, 2), h=(4e-9, 4e-9, 2e-9), o=(0, 0, 2e-9), Ms=6e5, K1=0.0,
                                           modules=1 | 2),
                                      dict(n=(1024, 1024, 1), h=(2e-9, 2e-9, 1.5e-9), o=(0, 0, 7e-9), Ms=1.1e6,
                                           K1=3e5, modules=1 | 2 | 8)],
                              A=1.5e-11, D=0.0, alpha=0.05, eval="RKDP54", dt=1e-14, tol=1e-5, init="sphere",
                              multilayer=0),
    # 256 independent films of uneven sizes advanced together, one launch per pass over all of them
    "batch256": dict(meshes=batch_systems(), A=1.3e-11, D=0.0, alpha=0.1, eval="RK4", dt=5e-14, init="sphere",
                     batched=True),
    # the batching workload with the demag field extrapolated quadratically between steps
    "batch256_es3": dict(meshes=batch_systems(), A=1.3e-11, D=0.0, alpha=0.1, eval="RK4", dt=5e-14, init="sphere",
                         batched=True, evalspeedup=3),
    # the same stack at half the in-plane size (FFT 1024 x 1024 x 4): small case for ncu captures
    "multilayer_stack3_512": dict(meshes=[dict(n=(512, 512, 1), h=(2e-9, 2e-9, 1e-9), o=(0, 0, 0), Ms=1.4e6, K1=0.0,
                                               modules=1 | 2),
                                          dict(n=(256, 256, 2), h=(4e-9, 4e-9, 2e-9), o=(0, 0, 2e-9), Ms=6e5, K1=0.0,
                                               modules=1 | 2),
                                          dict(n=(512, 512, 1), h=(2e-9, 2e-9, 1.5e-9), o=(0, 0, 7e-9), Ms=1.1e6,
                                               K1=3e5, modules=1 | 2 | 8)],
                                  A=1.5e-11, D=0.0, alpha=0.05, eval="RKDP54", dt=1e-14, tol=1e-5, init="sphere",
                                  multilayer=0),
}
MU0 = 1.256637061435916e-6
# seconds of timed CPU-reference steps after which the reference arm stops (whole steps of the full
# film take several seconds each on the host)
REF_TIME_CAP = 150



# DRAM traffic per cell of one launch of the roofline kernel (dram__bytes_read.sum +
# dram__bytes_write.sum of one ncu capture on the half-size case, divided by its cells;
# profiles/stage_rx16_lo_film3d_512x512x8.md, profiles/zmid_ml_multilayer_stack3_512.md)
TRAFFIC_PER_CELL = {("film3d", "stage"): (201.792e6 + 61.450496e6) / (512 * 512 * 8),
                    ("multilayer", "ml_zmid"): 383.30e6 / (512 * 512 + 256 * 256 * 2 + 512 * 512)}


def adjoint_problem(seed=4):
    """The differentiation workload: film 256 x 256 x 1 of 4 x 4 x 3 nm; Ms map 8e5 (1 + 0.1 g), g a
    unit-variance Gaussian random field of 20 nm correlation length (white noise filtered by
    exp(-k^2 l^2 / 4) in Fourier space, seeded); K1 map ~ U[0, 2e5] along z; A = 1.3e-11, alpha = 0.02;
    64 piecewise-constant field samples ~ N(0, 5e3^2) per component over 1 ns; m0 = +z tilted by up
    to 15 degrees; target = random unit vectors (seeded); RK4 dt = 1e-13, 10000 steps, checkpoint
    every 100."""
    rng = np.random.default_rng(seed)
    nx = ny = 256
    h = 4e-9
    white = rng.normal(size=(ny, nx))
    kx = 2 * np.pi * np.fft.fftfreq(nx, d=h)
    ky = 2 * np.pi * np.fft.fftfreq(ny, d=h)
    k2 = ky[:, None] ** 2 + kx[None, :] ** 2
    g = np.real(np.fft.ifft2(np.fft.fft2(white) * np.exp(-k2 * (20e-9) ** 2 / 4)))
    g = (g - g.mean()) / g.std()
    Ms = 8e5 * (1 + 0.1 * g.reshape(-1))
    K1 = rng.uniform(0, 2e5, nx * ny)
    Ha = rng.normal(0, 5e3, (64, 3))
    th = np.deg2rad(rng.uniform(0, 15.0, nx * ny))
    ph = rng.uniform(0, 2 * np.pi, nx * ny)
    m0 = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=1)
    t = rng.normal(size=(nx * ny, 3))
    t /= np.linalg.norm(t, axis=1)[:, None]
    return dict(n=(nx, ny, 1), h=(h, h, 3e-9), Ms=Ms, K1=K1, Ha=Ha, t_span=1e-9, m0=m0, target=t, A=1.3e-11,
                alpha=0.02, dt=1e-13, steps=10000, ckpt=100)


def adjoint_rate(bm, prec, device, steps=None):
    """Forward and backward device time of the differentiation workload (gradients of the loss
    with respect to the Ms map, K1 map and field samples)."""
    p = adjoint_problem()
    steps = steps or p["steps"]
    c = bm.Context(device=device, precision=prec)
    c.add_mesh(p["n"], p["h"])
    c.set_material(0, Ms=8e5, A=p["A"], alpha=p["alpha"], ea=(0, 0, 1))
    c.set_material_maps(0, Ms_map=p["Ms"], K1_map=p["K1"])
    c.set_modules(0, 1 | 2 | 8 | 16)
    c.set_field(0, p["Ha"], p["t_span"])
    c.setode("RK4", p["dt"])
    c.set_m(p["m0"] * p["Ms"][:, None])
    c.run(2)                                   # warm-up: kernels, tiles, graph
    c.set_m(p["m0"] * p["Ms"][:, None])
    loss, dMs, dK1, dHa, (f_ms, b_ms) = c.adjoint_rk4(p["target"], steps, p["ckpt"], True, nHa=64)
    c.close()
    ncell = p["n"][0] * p["n"][1]
    return {"workload": "adjoint_film256 (RK4, %d steps, checkpoint every %d)" % (steps, p["ckpt"]), "loss": loss,
            "forward_ms": f_ms, "backward_ms": b_ms, "adjoint_over_forward": b_ms / f_ms,
            "forward_Mcell_steps_per_s": ncell * steps / (f_ms * 1e-3) / 1e6,
            "grad_norms": {"Ms": float(np.linalg.norm(dMs)), "K1": float(np.linalg.norm(dK1)),
                           "Ha": float(np.linalg.norm(dHa))}}


def nice(n):
    b = 1
    while b < n:
        b *= 2
    t = 3
    while t < b:
        if t >= n:
            return t
        t *= 2
    return b


def rk4_step_bytes(cfg, p):
    """Algorithmic bytes of one RK4 step over every mesh (p bytes per real): per evaluation the y
    passes, z pass with its kernel read and the stage kernel's S1 rows (2D: the fused y pass), per
    step 19 cell-vector reads/writes of the stage updates (M in, base, rhs out, M out each stage,
    plus the three earlier rhs of the last stage)."""
    R, C = 3 * p, 6 * p
    tot = 0.0
    for m in mesh_list(cfg):
        nx, ny, nz = m["n"]
        Nx, Ny = 2 * nice(nx), 2 * nice(ny)
        Nz = 2 * nice(nz) if nz > 1 else 1
        LX = Nx // 2
        S1, S2 = LX * ny * nz, LX * Ny * nz
        if nz > 1:
            demag = 2 * C * (S1 + S2) + 2 * C * S2 + 6 * p * (LX + 1) * (Ny // 2 + 1) * (Nz // 2 + 1)
        else:
            demag = 2 * C * S1 + 4 * p * (LX + 1) * (Ny // 2 + 1)
        tot += 4 * (demag + 2 * C * S1) + 19 * R * nx * ny * nz
    return tot


def mesh_list(cfg):
    """The meshes of a workload as dicts with n, h, o, Ms, K1, modules."""
    if "meshes" in cfg:
        return cfg["meshes"]
    return [dict(n=cfg["n"], h=cfg["h"], o=(0, 0, 0), Ms=cfg["Ms"], K1=cfg["K1"], modules=cfg["modules"])]


def total_cells(cfg):
    return sum(m["n"][0] * m["n"][1] * m["n"][2] for m in mesh_list(cfg))


def init_all(cfg, seed):
    return [init_m(dict(cfg, n=m["n"], Ms=m["Ms"]), seed + 101 * q) for q, m in enumerate(mesh_list(cfg))]


def init_m(cfg, seed):
    n = cfg["n"][0] * cfg["n"][1] * cfg["n"][2]
    rng = np.random.default_rng(seed)
    if cfg["init"] == "tilt":
        th = np.deg2rad(rng.uniform(0.0, 15.0, n))
        ph = rng.uniform(0.0, 2 * np.pi, n)
        v = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=1)
    else:
        v = rng.normal(size=(n, 3))
        v /= np.linalg.norm(v, axis=1)[:, None]
    return np.ascontiguousarray(v * cfg["Ms"])


def make_ctx(bm, cfg, device, precision):
    c = bm.Context(device=device, precision=precision)
    for q, m in enumerate(mesh_list(cfg)):
        c.add_mesh(m["n"], m["h"], m["o"])
        c.set_material(q, Ms=m["Ms"], A=m.get("A", cfg["A"]), alpha=m.get("alpha", cfg["alpha"]),
                       grel=cfg.get("grel", 1.0), K1=m["K1"], ea=(0, 0, 1), D=cfg["D"])
        c.set_modules(q, m["modules"])
        c.set_field(q, cfg.get("Ha", (0, 0, 0)))
    if "multilayer" in cfg:
        c.multiconvolution(cfg["multilayer"])
    if cfg.get("batched"):
        c.set_batched(True)
    c.setode(cfg["eval"], cfg["dt"])
    if cfg["eval"] == "RKDP54":
        c.astepctrl(cfg["tol"], 2.0, 1e-15, 3e-12)
    if cfg.get("evalspeedup"):
        c.evalspeedup(cfg["evalspeedup"])
    return c


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

        def run():
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.samples.append([x.strip() for x in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and s[3 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def ml_sample(cfg, shrink=4):
    """A bounded CPU sample of a multilayer workload: every mesh shrunk in-plane by `shrink`."""
    out = []
    for m in cfg["meshes"]:
        out.append(((m["n"][0] // shrink, m["n"][1] // shrink, m["n"][2]), tuple(m["h"]), tuple(m["o"])))
    return out


def cpu_reference_ml(cfg, warmup, evals):
    """Seconds per H_demag evaluation of the reference's multilayered convolution
    (DemagKernelCollection + VEC mesh transfer, compiled CPU build) on the shrunk sample."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_libs import reference, MultiLayer
    if reference() is None:
        return None, None
    sample = ml_sample(cfg)
    ml = MultiLayer(sample, cfg["multilayer"], which="reference")
    n = sum(a[0][0] * a[0][1] * a[0][2] for a in sample)
    rng = np.random.default_rng(7)
    M = rng.normal(size=(n, 3))
    M = M / np.linalg.norm(M, axis=1)[:, None] * 1e6
    times = []
    for i in range(warmup + evals):
        t0 = time.perf_counter()
        ml.eval(M)
        if i >= warmup:
            times.append(time.perf_counter() - t0)
    ml.close()
    return float(np.mean(times)), sample


def reference_film_solver(cfg, seed=7):
    """The CPU reference of a single-film workload: the film's full field-and-integrate step with the
    demag convolution and the exchange / iDMI stencils from the reference's own compiled sources
    (oracle/_ref: Convolution<DemagKernel>, VEC_VC stencils, project FFTW-API shim) and Zeeman,
    uniaxial anisotropy, LLG and the RK4 / RKDP54 stages and step control from the oracle
    restatement (oracle/oracle.c), all OpenMP over the host's cores. Returns (solver, setup_s) or
    (None, reason)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_libs import OracleSolver, reference
    if reference() is None:
        return None, "reference CPU build (oracle/_ref) not present"
    t0 = time.perf_counter()
    mesh = dict(n=cfg["n"], h=cfg["h"], Ms=cfg["Ms"], A=cfg["A"], D=cfg["D"], K1=cfg["K1"], alpha=cfg["alpha"],
                grel=cfg.get("grel", 1.0), modules=cfg["modules"], Ha=cfg.get("Ha", (0, 0, 0)))
    ev = 1 if cfg["eval"] == "RKDP54" else 0
    s = OracleSolver([mesh], evaluation=ev, dt=cfg["dt"], tol=cfg.get("tol", 1e-5), dT_incr=2.0, dT_min=1e-15,
                     dT_max=3e-12)
    s.use_reference_fields(0)
    s.set_m(init_m(cfg, seed))
    return s, time.perf_counter() - t0


def reference_film_steps(s, warmup, steps, time_cap):
    """Time whole steps of the CPU reference solver: `warmup` untimed, then up to `steps` timed
    ones, stopping early once `time_cap` seconds of timed steps have run. Returns (steps run,
    seconds, field evaluations)."""
    if warmup:
        s.run(warmup)
    st0 = s.run(0)
    done, tsum = 0, 0.0
    while done < steps and tsum < time_cap:
        t0 = time.perf_counter()
        s.run(1)
        tsum += time.perf_counter() - t0
        done += 1
    st1 = s.run(0)
    return done, tsum, st1["evals"] - st0["evals"]


def cpu_reference_rate(cfg, steps=2):
    """cpu_baseline of a single-film workload: whole steps of the CPU reference (reference_film_solver)
    on the full film. Multilayer workloads: the reference's multilayered convolution alone on a
    shrunk sample (cpu_reference_ml)."""
    if "meshes" in cfg:
        if "multilayer" not in cfg:
            return {"error": "no CPU reference for batched independent meshes"}
        dt, sample = cpu_reference_ml(cfg, 1, 2)
        if dt is None:
            return {"error": "reference CPU build (oracle/_ref) not present"}
        n = sum(a[0][0] * a[0][1] * a[0][2] for a in sample)
        per_step = 6 if cfg["eval"] == "RKDP54" else 4
        return {"value": n / (per_step * dt) / 1e6, "unit": "Mcell-steps/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "reference CPU multilayered convolution alone (SDemag multilayer: DemagKernelCollection + "
                          "weighted mesh transfer, project FFTW-API shim) on the meshes shrunk 4x in-plane %s, 2 "
                          "evaluations, counted as %d per step; other field terms and stages not timed"
                          % ([a[0] for a in sample], per_step), "sec_per_eval": dt}
    s, setup = reference_film_solver(cfg)
    if s is None:
        return {"error": setup}
    done, tsum, evals = reference_film_steps(s, 0, steps, 1e9)
    s.close()
    ncell = total_cells(cfg)
    return {"value": ncell * done / tsum / 1e6, "unit": "Mcell-steps/s", "cores": os.cpu_count(), "kind": "reference",
            "sample": "%d whole %s steps (%d field evaluations) of the full %s film: demag convolution and %s "
                      "stencils from the reference's compiled sources (project FFTW-API shim), Zeeman, "
                      "anisotropy, LLG and stages from the oracle restatement; setup (kernel build) %.1f s "
                      "not timed" % (done, cfg["eval"], evals, "x".join(map(str, cfg["n"])),
                                     "iDMI+exchange" if cfg["modules"] & 4 else "exchange", setup),
            "sec_per_step": tsum / done}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0, None
    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    import datetime
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return rank, ws, local, dist


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="film3d_512x512x16", choices=sorted(CONFIGS))
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="timed steps only (for profiler launch lists)")
    ap.add_argument("--reference-gpu-bar", action="store_true",
                    help="only the same-box reference GPU bar of the workload (for profiler launch lists)")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    ncell = total_cells(cfg)
    rank, ws, local, dist = dist_setup()
    base = {"metric": "Mcell-steps/s", "unit": "Mcell-steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "data": "synthetic (seeded initial magnetization, random-init state of the named film)",
            "config": {"workload": args.config, "cells": [list(m["n"]) for m in mesh_list(cfg)],
                       "cellsize_m": [list(m["h"]) for m in mesh_list(cfg)],
                       "evaluation": cfg["eval"], "modules": [m["modules"] for m in mesh_list(cfg)],
                       "parallelism": "replicas x%d" % ws,
                       "l2": "working set above L2 (126 MB) every step"}}

    if args.impl == "reference":
        if rank != 0:
            if dist:
                dist.barrier()
                dist.destroy_process_group()
            return
        vals = []
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from oracle_libs import reference, dp, P
        R = reference()
        if R is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) not present"}))
            return
        per_step = 6 if cfg["eval"] == "RKDP54" else 4
        if "meshes" in cfg:
            dt, sample = cpu_reference_ml(cfg, args.warmup, args.steps)
            nsc = sum(a[0][0] * a[0][1] * a[0][2] for a in sample)
            v = nsc / (dt * per_step) / 1e6
            out = dict(base, impl="reference", value=v, ms_per_step=dt * per_step * 1e3, dtype="f64",
                       cpu_baseline={"value": v, "unit": "Mcell-steps/s", "cores": os.cpu_count(), "kind": "reference",
                                     "sample": "each step = %d evaluations of the reference CPU multilayered convolution "
                                               "on the meshes shrunk 4x in-plane %s" % (per_step, [a[0] for a in sample])},
                       e2e={"value": v, "unit": "Mcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
            print(json.dumps(out))
            return
        # the whole film, whole steps: the reference's compiled demag convolution and exchange / iDMI
        # stencils with the restated Zeeman, anisotropy, LLG and RK stages (reference_film_solver).
        # One warm-up step (the host path has no kernels or graphs to build); timed steps stop at
        # --steps or after REF_TIME_CAP seconds, and "steps" reports the number actually run.
        solver, setup = reference_film_solver(cfg)
        if solver is None:
            print(json.dumps({"impl": "reference", "unavailable": setup}))
            return
        done, tsum, evals = reference_film_steps(solver, min(args.warmup, 1), args.steps, REF_TIME_CAP)
        solver.close()
        tstep = tsum / done
        v = ncell / tstep / 1e6
        sample = ("each step = one whole %s step (%d field evaluations in %d steps) of the full %s film: demag "
                  "convolution and %s stencils from the reference's compiled sources (project FFTW-API shim), "
                  "Zeeman, uniaxial anisotropy, LLG and stage updates from the oracle restatement; %d timed steps "
                  "of %d asked (time cap %d s); kernel build %.1f s not timed"
                  % (cfg["eval"], evals, done, "x".join(map(str, cfg["n"])),
                     "iDMI+exchange" if cfg["modules"] & 4 else "exchange", done, args.steps, REF_TIME_CAP, setup))
        out = dict(base, impl="reference", value=v, ms_per_step=tstep * 1e3, dtype="f64", steps=done,
                   steps_requested=args.steps, warmup=min(args.warmup, 1),
                   cpu_baseline={"value": v, "unit": "Mcell-steps/s", "cores": os.cpu_count(), "kind": "reference",
                                 "sample": sample},
                   e2e={"value": v, "unit": "Mcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        print(json.dumps(out))
        return

    import boris2_b200 as bm
    if args.reference_gpu_bar:
        if rank == 0:
            print(json.dumps(dict(base, reference_gpu=reference_gpu_bar(bm, cfg, local, reps=args.steps))))
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    prec = bm.MIXED if args.precision == "mixed" else bm.FP64
    c = make_ctx(bm, cfg, local, prec)
    M0 = init_all(cfg, 1234 + rank)
    for q, Mq in enumerate(M0):
        c.set_m(Mq, q)
    # warm-up (also builds kernels and the CUDA graph)
    c.run(args.warmup)
    c.sync()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    st0 = c.stats()
    st, ms = c.run_timed(args.steps)
    clocks = sampler.stop()
    if dist:
        import torch
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    steps_done = st["accepted"] - st0["accepted"]
    value = ncell * steps_done * ws / (ms * 1e-3) / 1e6
    attempts = st["attempts"] - st0["attempts"]
    if args.no_extras:
        if rank == 0:
            print(json.dumps(dict(base, value=value, ms_per_step=ms / max(steps_done, 1), note="no extras")))
        c.close()
        return
    # e2e through the C ABI with host buffers (pinned), copies inside the timed region
    bufs = []
    for Mq in M0:
        try:
            import torch
            Mpin = torch.from_numpy(Mq.reshape(-1).copy()).pin_memory()
            Mout = torch.empty_like(Mpin).pin_memory()
            bufs.append((Mpin.numpy(), Mout.numpy(), Mpin, Mout))
        except Exception:
            bufs.append((Mq.reshape(-1).copy(), np.empty(Mq.size), None, None))
    c.sync()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for q, bq in enumerate(bufs):
        c.set_m(bq[0], q)
    st1 = c.stats()
    st2 = c.run(args.steps)
    for q, bq in enumerate(bufs):
        c.get_m(q, out=bq[1])
    e2e_s = time.perf_counter() - t0
    if dist:
        import torch
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_steps = st2["accepted"] - st1["accepted"]
    e2e = ncell * e2e_steps * ws / e2e_s / 1e6
    # kernel timing for the roofline: dominant kernel of one field evaluation
    peak, peak_kind = peaks()
    ml = "multilayer" in cfg
    if cfg.get("batched"):
        # one launch per pass over every system: the roofline is that of the whole step
        p = 4 if prec == bm.MIXED else 8
        kbytes = np.array([rk4_step_bytes(cfg, p)])
        kms = np.array([ms / max(steps_done, 1)])
        names = ["batched RK4 step (all passes, all systems)"]
        dom = 0
        kernels = {names[0]: {"ms": kms[0], "GB/s": kbytes[0] / (kms[0] * 1e-3) / 1e9}}
        tiles = None
    elif ml:
        kms, kbytes = c.ml_time_kernels(reps=10)
        names = ["ml_transfer_in_xfwd", "ml_yfwd", "ml_zmid", "ml_yinv", "ml_xinv_transfer_out"]
        dom = int(np.argmax(kms[:5]))
        kernels = {names[i]: {"ms": kms[i], "GB/s": kbytes[i] / (kms[i] * 1e-3) / 1e9} for i in range(5) if kms[i] > 0}
        kernels["demag_evaluation"] = {"ms": kms[5], "GB/s": kbytes[5] / (kms[5] * 1e-3) / 1e9,
                                       "frac": kbytes[5] / (kms[5] * 1e-3) / 1e9 / peak}
        tiles = {"zmid_ml_W": c.ml_tile()}
    else:
        # every launch of a few eager steps timed one by one (the step graph's launches, buffers and
        # arguments), summed per kernel kind with each launch's algorithmic bytes
        tk = c.time_step(steps=3)
        names = [k for k in tk if k != "other"]
        kms = np.array([tk[k]["ms"] / tk[k]["launches"] for k in names])
        kbytes = np.array([tk[k]["bytes"] / tk[k]["launches"] for k in names])
        dom = int(np.argmax([tk[k]["ms"] for k in names]))
        kernels = {k: {"ms_per_launch": tk[k]["ms"] / tk[k]["launches"], "launches": tk[k]["launches"],
                       "GB/s": (tk[k]["bytes"] / (tk[k]["ms"] * 1e-3) / 1e9 if tk[k]["bytes"] else None)}
                   for k in tk}
        tot_b = sum(tk[k]["bytes"] for k in tk)
        tot_ms = sum(tk[k]["ms"] for k in tk)
        kernels["all_launches"] = {"ms": tot_ms, "GB/s": tot_b / (tot_ms * 1e-3) / 1e9,
                                   "frac": tot_b / (tot_ms * 1e-3) / 1e9 / peak,
                                   "timing": "3 eager steps, CUDA event after every launch"}
        tiles = c.tiles(0)
    achieved = kbytes[dom] / (kms[dom] * 1e-3) / 1e9
    tpc = TRAFFIC_PER_CELL.get(("multilayer" if ml else "film3d", names[dom]))
    traffic = tpc * ncell if (tpc and (ml or args.config.startswith("film3d"))) else None
    kpe = c.kernels_per_step()
    out = dict(base, value=value, ms_per_step=ms / max(steps_done, 1), dtype="f32" if prec == bm.MIXED else "f64",
               e2e={"value": e2e, "unit": "Mcell-steps/s", "h2d_bytes_per_step": 3 * ncell * 8 / max(e2e_steps, 1),
                    "d2h_bytes_per_step": 3 * ncell * 8 / max(e2e_steps, 1)},
               gpu_launches=int(kpe * attempts if cfg["eval"] == "RKDP54" else kpe * steps_done),
               clocks=clocks,
               roofline={"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak,
                         "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "algorithmic_bytes_per_launch": kbytes[dom],
                         "launch_ms": kms[dom],
                         "timing": ("launches inside eager steps of the workload (CUDA events on the "
                                    "context's stream between launches)" if not (ml or cfg.get("batched"))
                                    else "per-part launches (multilayer) or whole steps (batched)")},
               kernels=kernels,
               rkdp={"attempts": attempts, "accepted": steps_done, "dT": st["dT"]})
    if tiles:
        out["tiles"] = tiles
    c.close()
    if rank == 0 and ws == 1:
        extra_steps = max(3, min(args.steps, 10))
        # the same workload in the FP64 plain form
        if prec == bm.MIXED:
            try:
                f = quick_rate(bm, cfg, bm.FP64, extra_steps, args.warmup, local)
                out["fp64_plain"] = dict(f, speedup_mixed_over_fp64=value / f["value"])
            except Exception as e:
                out["fp64_plain"] = {"error": str(e)}
        # the multilayered convolution workload (three stacked meshes), mixed and FP64
        if not ml and args.config == "film3d_512x512x16":
            try:
                mcfg = CONFIGS["multilayer_stack3"]
                mx = quick_rate(bm, mcfg, bm.MIXED, extra_steps, args.warmup, local, ml_timing=True)
                f64 = quick_rate(bm, mcfg, bm.FP64, extra_steps, args.warmup, local, ml_timing=True)
                out["multilayer"] = {"workload": "multilayer_stack3", "cells": total_cells(mcfg), "mixed": mx,
                                     "fp64_plain": f64, "speedup_mixed_over_fp64": mx["value"] / f64["value"],
                                     "peak_GB/s": peak}
            except Exception as e:
                out["multilayer"] = {"error": str(e)}
        # the batching workload (256 uneven films, one launch per pass over all of them)
        if not ml and args.config == "film3d_512x512x16":
            try:
                bcfg = CONFIGS["batch256"]
                bx = quick_rate(bm, bcfg, bm.MIXED, 5, 2, local)
                pb = rk4_step_bytes(bcfg, 4)
                bes = quick_rate(bm, CONFIGS["batch256_es3"], bm.MIXED, 5, 3, local)
                out["batching"] = {"workload": "batch256", "systems": len(bcfg["meshes"]), "cells": total_cells(bcfg),
                                   "mixed": bx, "mixed_evalspeedup_quadratic": bes,
                                   "step_GB/s": pb / (bx["ms_per_step"] * 1e-3) / 1e9,
                                   "step_frac_of_peak": pb / (bx["ms_per_step"] * 1e-3) / 1e9 / peak}
            except Exception as e:
                out["batching"] = {"error": str(e)}
        # evaluation speedup: the same film under RK4 (dt 1e-14), plain and with the demag field
        # extrapolated quadratically between steps
        if not ml and args.config == "film3d_512x512x16":
            try:
                rk = dict(cfg, eval="RK4")
                plain = quick_rate(bm, rk, bm.MIXED, extra_steps, args.warmup, local)
                es3 = quick_rate(bm, dict(rk, evalspeedup=3), bm.MIXED, extra_steps + 3, args.warmup, local)
                dp3 = quick_rate(bm, dict(cfg, evalspeedup=3), bm.MIXED, extra_steps + 3, args.warmup, local)
                out["evalspeedup"] = {"workload": "film3d_512x512x16 RK4 dt 1e-14 / RKDP54 tol 1e-5", "rk4_plain": plain,
                                      "rk4_quadratic": es3, "speedup": es3["value"] / plain["value"],
                                      "rkdp54_quadratic": dp3, "rkdp54_speedup": dp3["value"] / value}
            except Exception as e:
                out["evalspeedup"] = {"error": str(e)}
        # the differentiation workload: adjoint / forward device time
        if not ml and args.config == "film3d_512x512x16":
            try:
                out["adjoint"] = adjoint_rate(bm, bm.MIXED, local)
            except Exception as e:
                out["adjoint"] = {"error": str(e)}
        # precision against FP64: the GPU FP64 plain form and the reference's CPU build, on the
        # same seeded M, at the workload's full size
        if not ml and not cfg.get("batched"):
            try:
                out["precision"] = precision_film(bm, cfg, local, with_reference=not args.no_cpu_baseline)
                cb = out["precision"].pop("_cpu_baseline", None)
                if cb is not None:
                    out["cpu_baseline"] = cb
            except Exception as e:
                out["precision"] = {"error": str(e)}
        if not ml and not cfg.get("batched"):
            try:
                out["reference_gpu"] = reference_gpu_bar(bm, cfg, local)
                if "mixed" in out["reference_gpu"]:
                    out["vs_ref_gpu_demag"] = out["reference_gpu"]["mixed"]["speedup"]
            except Exception as e:
                out["reference_gpu"] = {"error": str(e)}
        if not args.no_cpu_baseline and "cpu_baseline" not in out:
            try:
                out["cpu_baseline"] = cpu_reference_rate(cfg)
            except Exception as e:  # reported, not fatal
                out["cpu_baseline"] = {"error": str(e)}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def rel_err(a, ref):
    """max and RMS over cells of |a - ref| / max |ref| (vector norms per cell)."""
    d = np.linalg.norm(np.asarray(a).reshape(-1, 3) - np.asarray(ref).reshape(-1, 3), axis=1)
    s = np.linalg.norm(np.asarray(ref).reshape(-1, 3), axis=1).max()
    return {"max": float(d.max() / s), "rms": float(np.sqrt(np.mean(d * d)) / s)}


def precision_film(bm, cfg, device, with_reference=True, ref_steps=2, gpu_steps=5000):
    """Errors of the mixed-precision path (and of the GPU FP64 plain form) against FP64 on the
    workload's full film, from one seeded M:
      h_demag            H_demag of M: mixed and GPU FP64 against the reference's CPU build
                         (Convolution<DemagKernel>), and mixed against GPU FP64; relative to max |H_ref|
      m_after_ref_steps  m after `ref_steps` whole steps of the workload's stepper from M: mixed and GPU
                         FP64 against the CPU reference solver (reference_film_solver); |dm| per cell
      m_after_gpu_steps  m after `gpu_steps` steps (the workload's run length): mixed against GPU FP64,
                         and their simulated times
    Tolerances stated by the workload: 1e-5 on H_demag, 1e-4 on |dm|. The CPU reference steps are also
    timed and returned as the cpu_baseline (key _cpu_baseline)."""
    M = init_m(cfg, 4321)
    ms = cfg["Ms"]
    res = {"tolerance": {"h_demag_rel": 1e-5, "dm_abs": 1e-4}, "seed_m": 4321}
    Hd, mref, mgpu, tgpu = {}, {}, {}, {}
    for name, prec in (("mixed", bm.MIXED), ("fp64", bm.FP64)):
        c = make_ctx(bm, cfg, device, prec)
        c.set_m(M)
        Hd[name] = c.demag_field()
        c.set_m(M)
        c.run(ref_steps)
        mref[name] = c.get_m() / ms
        c.set_m(M)
        st = c.run(gpu_steps)
        mgpu[name] = c.get_m() / ms
        tgpu[name] = st["time"]
        c.close()
    res["h_demag"] = {"mixed_vs_fp64_gpu": rel_err(Hd["mixed"], Hd["fp64"])}
    dmg = np.linalg.norm(mgpu["mixed"] - mgpu["fp64"], axis=1)
    res["m_after_gpu_steps"] = {"steps": gpu_steps, "evaluation": cfg["eval"],
                                "mixed_vs_fp64_gpu": {"max": float(dmg.max()), "rms": float(np.sqrt(np.mean(dmg ** 2)))},
                                "time_s": {"mixed": tgpu["mixed"], "fp64": tgpu["fp64"]}}
    if with_reference:
        solver, setup = reference_film_solver(dict(cfg), seed=0)
        if solver is None:
            res["reference"] = {"error": setup}
            return res
        Href = solver.reference_hdemag(M)
        res["h_demag"]["mixed_vs_reference_cpu"] = rel_err(Hd["mixed"], Href)
        res["h_demag"]["fp64_gpu_vs_reference_cpu"] = rel_err(Hd["fp64"], Href)
        solver.set_m(M)
        done, tsum, evals = reference_film_steps(solver, 0, ref_steps, 1e9)
        mr = solver.get_m() / ms
        solver.close()
        blk = {"steps": done, "evaluation": cfg["eval"]}
        for name in ("mixed", "fp64"):
            d = np.linalg.norm(mref[name] - mr, axis=1)
            blk[name + "_vs_reference_cpu"] = {"max": float(d.max()), "rms": float(np.sqrt(np.mean(d * d)))}
        res["m_after_ref_steps"] = blk
        ncell = total_cells(cfg)
        res["_cpu_baseline"] = {
            "value": ncell * done / tsum / 1e6, "unit": "Mcell-steps/s", "cores": os.cpu_count(), "kind": "reference",
            "sample": "%d whole %s steps (%d field evaluations) of the full %s film from the precision block's M: "
                      "demag convolution and %s stencils from the reference's compiled sources (project FFTW-API "
                      "shim), Zeeman, anisotropy, LLG and stages from the oracle restatement; kernel build %.1f s "
                      "not timed" % (done, cfg["eval"], evals, "x".join(map(str, cfg["n"])),
                                     "iDMI+exchange" if cfg["modules"] & 4 else "exchange", setup),
            "sec_per_step": tsum / done}
    return res


def reference_gpu_bar(bm, cfg, device, reps=20):
    """The same-box reference GPU bar: one H_demag evaluation of the workload's film by the reference's
    own GPU convolution (ConvolutionCUDA<., DemagKernelCUDA>: cuFFT plans, transposes and its fused
    q2D z-product kernels, built unmodified for sm_100a by baseline/Makefile) in FP32 and FP64, against
    one evaluation of this path (bm_time_demag: x transform, y / z passes, inverse x), device time
    with CUDA events, plus the two fields' difference on the same M."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_libs import reference_gpu, ReferenceGPUDemag
    M = init_m(cfg, 4321)
    out = {"reps": reps}
    for name, ours, refp in (("mixed", bm.MIXED, "f32"), ("fp64", bm.FP64, "f64")):
        if reference_gpu(refp) is None:
            return {"error": "reference GPU build (baseline/_ref) not present"}
        c = make_ctx(bm, cfg, device, ours)
        c.set_m(M)
        H = c.demag_field()
        t_ours = c.time_demag(0, reps)
        c.close()
        g = ReferenceGPUDemag(cfg["n"], cfg["h"], refp)
        Hr = g.field(M)
        t_ref = g.time(reps)
        g.close()
        out[name] = {"ours_ms_per_eval": t_ours, "reference_gpu_ms_per_eval": t_ref,
                     "reference_gpu_precision": refp, "speedup": t_ref / t_ours,
                     "h_demag_vs_reference_gpu": rel_err(H, Hr)}
    return out


def quick_rate(bm, cfg, prec, steps, warmup, device, ml_timing=False):
    """Mcell-steps/s of a workload over a short device-timed run (plus the multilayer demag
    evaluation time and algorithmic GB/s when asked)."""
    c = make_ctx(bm, cfg, device, prec)
    for q, Mq in enumerate(init_all(cfg, 4321)):
        c.set_m(Mq, q)
    c.run(warmup)
    c.sync()
    st0 = c.stats()
    st, ms = c.run_timed(steps)
    done = st["accepted"] - st0["accepted"]
    r = {"value": total_cells(cfg) * done / (ms * 1e-3) / 1e6, "ms_per_step": ms / max(done, 1), "steps": done,
         "attempts": st["attempts"] - st0["attempts"]}
    if ml_timing:
        kms, kb = c.ml_time_kernels(reps=5)
        r["demag_evaluation_ms"] = kms[5]
        r["demag_GB/s"] = kb[5] / (kms[5] * 1e-3) / 1e9
        r["zmid_ml_ms"] = kms[2]
        r["zmid_ml_GB/s"] = kb[2] / (kms[2] * 1e-3) / 1e9
    c.close()
    return r


if __name__ == "__main__":
    main()
