"""Benchmark of the CUDA path tracer on the BVH-stress workload.

Workload: a 2^20-triangle UV sphere (1024 x 512, vertices displaced radially by seeded gradient
noise of 5 % amplitude) inside a closed Lambertian box with one area light; 1920 x 1080 pinhole
camera; four hero wavelengths over 360-830 nm; max depth 12, Russian roulette from depth 6. The
scene is generated here (synthetic data; the reference ships no such scene).

One step is one pass of one sample per pixel: 2,073,600 camera paths. The metric is spectral paths
per second over the whole job; every rank renders its own sample streams of the same image (weak
scaling) and the films are summed over NCCL once at the end.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

`--impl reference` times the reference engine's own CPU transport (compiled from its sources into
oracle/_ref) on this machine's host cores over a bounded band of the same image.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "optical-pathtracer_b200")
sys.path.insert(0, PKG)

import owec_abi as A  # noqa: E402
import scenes  # noqa: E402

WIDTH, HEIGHT = 1920, 1080
MAX_DEPTH, RR_DEPTH = 12, 6
METRIC = "spectral paths/s"
def workload():
    return (f"bvh_stress_room: 2^20-tri displaced UV sphere in a Lambertian box, 1 area light, {WIDTH}x{HEIGHT}, "
            "hero-4 spectral, depth 12")
NODE_BYTES, PRIM_BYTES = 80, 48
RAY_STATE_BYTES = 4 + 64 + 24  # queue index, the path's ray record, the hit record written
# Arithmetic per visit, counted from the traversal's source: a wide node tests its 8 child boxes
# (per box 6 FMA-form plane distances = 12 flops, 6 min/max = 6, entry/exit compares = 6: 24), a
# triangle the shear-space watertight test and the plane distance (about 40).
NODE_FLOPS, PRIM_FLOPS = 8 * 24, 40


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


PRECISIONS = {"mixed": A.PRECISION_MIXED, "fp32": A.PRECISION_FP32, "fp64": A.PRECISION_FP64}
PRECISION = "mixed"


INTEGRATOR = "path"


def settings_for(rank):
    return A.make_settings(seed=rank, max_depth=MAX_DEPTH, rr_depth=RR_DEPTH, wavelength_mode=A.WAVELENGTHS_HERO4,
                           precision=PRECISIONS[PRECISION], integrator=INTEGRATOR)


def cpu_reference_rate(desc, seconds_target=12.0, threads=0):
    """The reference engine (oracle/_ref) on this host: paths/s over a band of image rows through
    the sphere, sized to about `seconds_target` of work. Returns (paths/s, threads, sample text)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_ref import ReferenceEngine  # the oracle, used here only as the timed CPU baseline
    ref = ReferenceEngine(desc)
    s = settings_for(0)
    # a probe band, then one sized to the target
    mid = HEIGHT // 2
    band = 8
    t0 = time.perf_counter()
    ref.render(s, 1, pixel_begin=(mid - band // 2) * WIDTH, pixel_end=(mid + band // 2) * WIDTH, threads=threads)
    dt = max(time.perf_counter() - t0, 1e-3)
    rows = int(min(HEIGHT, max(4, band * seconds_target / dt)))
    r0 = max(0, mid - rows // 2)
    t0 = time.perf_counter()
    _, st = ref.render(s, 1, pixel_begin=r0 * WIDTH, pixel_end=(r0 + rows) * WIDTH, threads=threads)
    dt = time.perf_counter() - t0
    n_threads = threads if threads > 0 else os.cpu_count()
    return st["paths"] / dt, n_threads, f"{rows} centre rows of the {WIDTH}x{HEIGHT} frame at 1 spp ({st['paths']} paths, {dt:.1f} s)"


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    desc = scenes.bvh_stress_room(WIDTH, HEIGHT).desc()
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    try:
        from oracle_ref import ReferenceEngine, REF_LIB
        if not os.path.exists(REF_LIB):
            raise RuntimeError("oracle/_ref/liboweref.so was not built")
        ref = ReferenceEngine(desc)
    except BaseException as e:  # pytest.skip raises a BaseException subclass
        print(json.dumps({"impl": "reference", "unavailable": f"reference engine not built: {e}"}))
        return 0
    s = settings_for(0)
    mid = HEIGHT // 2
    # size a step to about 2-3 s of host work
    t0 = time.perf_counter()
    ref.render(s, 1, pixel_begin=(mid - 2) * WIDTH, pixel_end=(mid + 2) * WIDTH)
    dt = max(time.perf_counter() - t0, 1e-3)
    rows = int(min(HEIGHT, max(2, 4 * 2.5 / dt)))
    r0 = max(0, mid - rows // 2)
    for _ in range(args.warmup):
        ref.render(s, 1, pixel_begin=r0 * WIDTH, pixel_end=(r0 + rows) * WIDTH)
    paths = 0
    t0 = time.perf_counter()
    for k in range(args.steps):
        _, st = ref.render(s, 1, first_pass=k + 1, pixel_begin=r0 * WIDTH, pixel_end=(r0 + rows) * WIDTH)
        paths += st["paths"]
    dt = time.perf_counter() - t0
    rate = paths / dt
    cores = os.cpu_count()
    sample = f"{rows} centre rows of the {WIDTH}x{HEIGHT} frame at 1 spp per step"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "paths/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload(), "rows_per_step": rows},
        "cpu_baseline": {"value": rate, "unit": "paths/s", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": rate, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def rel_mse(img, ref):
    """The reference's relative MSE (docs/BENCHMARKS.md): mean((img - ref)^2 / (ref^2 + 0.01 mean(ref)^2))
    over pixels and XYZ channels."""
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 0.01 * np.mean(ref) ** 2)))


def precision_study(device, ref_rows=16, ref_spp=1024, spp=16, bias_spp=256):
    """The metric's RMSE half on the bench's own workload at 1920 x 1080: each precision
    instantiation (FP32 + selective FP64, plain FP32, all FP64) against the reference engine's FP64
    CPU transport (oracle/_ref), which renders ref_rows rows through the middle of the frame at
    ref_spp samples per pixel (another seed). Per mode: paths/s of a one-sample pass; relMSE of a
    `spp` render over the band; seconds to a relMSE of 1e-3 (seconds per sample x spp x relMSE /
    1e-3, as relMSE falls as 1 / spp for an unbiased estimator); the bias (mean signed error over the
    band's pixels at bias_spp, relative to the reference's mean, with its standard error); the
    transport statistics. speedup_at_equal_relmse: FP64's seconds to that relMSE over the mode's."""
    import owe_cuda
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_ref import ReferenceEngine  # the FP64 oracle image, not a timed leg
    desc = scenes.bvh_stress_room(WIDTH, HEIGHT).desc()
    r0 = HEIGHT // 2 - ref_rows // 2
    t0 = time.perf_counter()
    ref_img, ref_st = ReferenceEngine(desc).render(
        A.make_settings(seed=1000, max_depth=MAX_DEPTH, rr_depth=RR_DEPTH, wavelength_mode=A.WAVELENGTHS_HERO4), 1,
        passes=ref_spp, pixel_begin=r0 * WIDTH, pixel_end=(r0 + ref_rows) * WIDTH)
    ref_band = ref_img[r0:r0 + ref_rows]
    out = {"film": f"{WIDTH}x{HEIGHT}", "oracle": f"reference engine FP64 CPU transport, rows {r0}-{r0 + ref_rows - 1}, "
           f"{ref_spp} spp, other seed ({time.perf_counter() - t0:.0f} s)", "spp": spp, "bias_spp": bias_spp,
           "target_relmse": 1e-3}
    for name, prec in (("mixed", A.PRECISION_MIXED), ("fp32", A.PRECISION_FP32), ("fp64", A.PRECISION_FP64)):
        with owe_cuda.Context(device) as c:
            c.upload(desc)
            c.build_bvh()
            c.set_settings(A.make_settings(seed=7, max_depth=MAX_DEPTH, rr_depth=RR_DEPTH,
                                           wavelength_mode=A.WAVELENGTHS_HERO4, precision=prec))
            c.run_pass(1)  # warm-up: the mode's primitives and path buffers
            secs = []
            for _ in range(3):
                c.run_pass(1)
                secs.append(c.last_pass_timing()[0])
            sec_per_spp = min(secs)
            c.reset_film()
            c.run_pass(spp)
            img = c.resolve()[0][r0:r0 + ref_rows]
            rm = rel_mse(img, ref_band)
            c.reset_film()
            c.set_pass_index(1 << 16)
            c.run_pass(bias_spp)
            img_b = c.resolve()[0][r0:r0 + ref_rows]
            st = c.stats()
        diff = (img_b - ref_band)[..., 1].ravel()
        mean_ref = float(ref_band[..., 1].mean())
        out[name] = {"paths_per_s": WIDTH * HEIGHT / sec_per_spp, "relmse": rm,
                     "seconds_to_target": sec_per_spp * spp * rm / 1e-3,
                     "bias": float(diff.mean()) / mean_ref, "bias_se": float(diff.std() / np.sqrt(diff.size)) / mean_ref,
                     "inconsistencies_per_path": st["inconsistencies"] / max(1, st["paths"]),
                     "leaks_per_path": st["leaks"] / max(1, st["paths"]), "faults": st["device_faults"]}
    for name in ("mixed", "fp32"):
        out[name]["speedup_at_equal_relmse"] = out["fp64"]["seconds_to_target"] / out[name]["seconds_to_target"]
    out["reference_leaks"] = ref_st["leaks"]
    return out


def adjoint_study(device, n=256, bins=512, walks=1 << 24):
    """The metric's adjoint half at the differentiable caustic's size: a 256 x 256 heightfield
    (heights 0), a 512 x 512 wall, 2^24 walks per step; device seconds of the forward walks and of
    the adjoint replay."""
    import owe_cuda
    sb, info = scenes.caustic_slab_scene(n=n, wall_bins=bins)
    w = scenes.caustic_walk(info, seed=1)
    target = scenes.gaussian_blobs(bins, count=64, seed=3)
    with owe_cuda.Context(device) as c:
        c.upload(sb.desc())
        c.build_bvh()
        c.set_heightfield(info["heightfield"], info["thickness"], np.zeros((n, n)))
        fw, ad = [], []
        for _ in range(3):
            c.walk_reset()
            c.walk(w, 0, walks)
            fw.append(c.walk_timing()[0])
            img, _ = c.walk_resolve()
            g = 2 * (img - target * img.mean())
            c.walk_adjoint(w, 0, walks, g)
            ad.append(c.walk_timing()[1])
    f, a = min(fw), min(ad)
    return {"heightfield": f"{n}x{n}", "bins": f"{bins}x{bins}", "walks": walks, "forward_s": f, "adjoint_s": a,
            "adjoint_over_forward": a / f, "forward_walks_per_s": walks / f}


def c5_study(device, spp_timing=1024, steps=0, spp_step=8, width=1920, height=1080):
    """The large adjoint: the caustic room (a 1024 x 1024 heightfield PMMA panel, two displaced-sphere
    props of 2^20 triangles each, fog with sigma_s 0.5 / m, sigma_a 0.05 / m, Henyey-Greenstein g 0.8,
    one ceiling light), 1920 x 1080, depth 24. Device seconds of a forward pass (owec_pass) and of the
    path-replay adjoint (owec_path_adjoint) over the same spp_timing samples, their ratio, the device
    memory of each; then, when steps > 0, that many Adam steps toward a target film (c5_optimise)."""
    import torch
    import owe_cuda
    n = 1024
    sb, info = scenes.caustic_room(width=width, height=height, panel_n=n)
    desc = sb.desc()
    settings = A.make_settings(seed=11, max_depth=24, rr_depth=6, wavelength_mode=A.WAVELENGTHS_HERO4)
    out = {"film": f"{width}x{height}", "heightfield": f"{n}x{n}", "depth": 24, "spp": spp_timing}
    free0, total = torch.cuda.mem_get_info(device)
    with owe_cuda.Context(device) as c:
        c.set_settings(settings)
        c.upload(desc)
        c.build_bvh()
        c.set_heightfield(info["heightfield"], info["base_z"], np.zeros(n * n))
        out["triangles"] = c.bvh_info()["triangles"]
        c.run_pass(1)
        c.path_adjoint(0, 1, np.zeros((height, width, 3)))  # warm-up: buffers, the replay's stacks
        free1, _ = torch.cuda.mem_get_info(device)
        c.reset_film()
        c.set_pass_index(100)
        c.run_pass(spp_timing)
        fwd = c.last_pass_timing()[0]
        img, _ = c.resolve(samples=False)
        g = np.zeros_like(img)
        g[..., 1] = 1.0 / img.size  # the gradient of the image's mean luminance
        _, st, _ = c.path_adjoint(100, spp_timing, g, with_stats=True)
        out.update({"forward_s": fwd, "adjoint_s": st["seconds"], "adjoint_over_forward": st["seconds"] / fwd,
                    "adjoint_replay_s": st["replay_seconds"],
                    "forward_paths_per_s": width * height * spp_timing / fwd,
                    "paths_met_heightfield": st["heightfield"] / max(1, st["paths"]),
                    "dropped_of_those": st["dropped"] / max(1, st["heightfield"]), "faults": st["faults"],
                    "context_bytes": int(free0 - free1), "adjoint_call_bytes": int(st["device_bytes"]),
                    "device_total_bytes": int(total)})
        if steps > 0:
            out["optimisation"] = c5_optimise(c, info, n, steps, spp_step, width, height)
    return out


def _bilinear(n, m):
    """The n x m matrix that samples a piecewise-linear function through m evenly spaced control
    values at n evenly spaced points (both ends included)."""
    x = np.linspace(0.0, m - 1.0, n)
    return np.maximum(0.0, 1.0 - np.abs(x[:, None] - np.arange(m)[None, :]))


def _screen_box(points, eye, look_at, up, fov_y_deg, width, height):
    """Pixel bounds (x0, x1, y0, y1) of world points seen by the pinhole observer (IdealObserver's
    image plane: x to the right, y down)."""
    eye, f = np.asarray(eye, float), np.asarray(look_at, float) - np.asarray(eye, float)
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, float))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    ty = np.tan(np.radians(fov_y_deg) / 2)
    tx = ty * width / height
    v = np.asarray(points, float) - eye
    px = (v @ r / (v @ f) / tx + 1) * width / 2
    py = (1 - v @ u / (v @ f) / ty) * height / 2
    return px.min(), px.max(), py.min(), py.max()


def c5_optimise(c, info, n, steps, spp_step, width, height, m=8, block=16, lr=2e-4):
    """Heightfield optimisation on the caustic room through owe_autograd.camera_film: the heights are
    a bilinear surface through an m x m grid of control heights (its outer ring held at zero, so the
    panel's rim stays flat), the target film is rendered at 64 spp at seeded target control heights,
    the loss is the mean squared difference of the two films averaged over block x block pixel
    tiles that show the panel (its outline projected to the screen, a tile wider on each side; the
    rest of the film does not depend on the heights and would add only its noise), and Adam steps
    the control heights (step size decaying tenfold over the run) with a gradient from an
    independent replay each step.
    The loss at 64 spp is measured before and after, beside the same loss between two independent
    64-spp renders at the target heights (the noise floor)."""
    import torch
    import torch.nn.functional as F
    import owe_autograd
    hf, base_z = info["heightfield"], info["base_z"]
    W = torch.from_numpy(_bilinear(n, m))
    rng = np.random.Generator(np.random.PCG64(5))
    u = np.linspace(0.0, 1.0, m)
    ct = np.zeros((m, m))
    for _ in range(4):
        fx, fy, px, py = rng.uniform(0.5, 2.0, 2).tolist() + rng.uniform(0, 2 * np.pi, 2).tolist()
        ct += np.outer(np.sin(np.pi * fy * u + py), np.sin(np.pi * fx * u + px))
    ct[0, :] = ct[-1, :] = ct[:, 0] = ct[:, -1] = 0
    ct *= 4e-3 / np.abs(ct).max()
    ct = torch.from_numpy(ct)
    mask = torch.zeros(m, m, dtype=torch.float64)
    mask[1:-1, 1:-1] = 1
    hc = height // block * block
    wc = width // block * block
    cx, cy, cz = info["centre"]
    half, thick = info["half"], info["thickness"]
    corners = [(cx + sx * half, cy + sy * half, cz + dz) for sx in (-1, 1) for sy in (-1, 1) for dz in (0.0, thick)]
    x0, x1, y0, y1 = _screen_box(corners, *info["view"], width, height)
    tx0, ty0 = max(0, int(x0 // block) - 1), max(0, int(y0 // block) - 1)
    tx1, ty1 = min(wc // block, int(x1 // block) + 2), min(hc // block, int(y1 // block) + 2)

    def heights(ctrl):
        return (W @ (ctrl * mask) @ W.T).reshape(-1)

    def tiles(img):
        x = img[:hc, :wc].permute(2, 0, 1).unsqueeze(0)
        return F.avg_pool2d(x, block)[..., ty0:ty1, tx0:tx1]

    def render(ctrl, first, spp):
        with torch.no_grad():
            return owe_autograd.camera_film(heights(ctrl), c, hf, base_z, first, spp)

    target = tiles(render(ct, 1 << 24, 64))
    def loss64(ctrl, first):
        return float(((tiles(render(ctrl, first, 64)) - target) ** 2).mean())

    ctrl = torch.zeros(m, m, dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([ctrl], lr=lr)
    decay = torch.optim.lr_scheduler.ExponentialLR(opt, gamma=0.1 ** (1.0 / steps))  # to lr / 10 at the end
    res = {"steps": steps, "spp_per_step": spp_step, "control_grid": f"{m}x{m} (outer ring fixed at 0)",
           "loss": f"mean squared XYZ difference of {block}x{block}-pixel tile means over the panel's "
                   f"{tx1 - tx0}x{ty1 - ty0} tiles", "adam_lr_m": lr,
           "loss64_noise_floor": loss64(ct, 1 << 25), "loss64_first": loss64(ctrl.detach(), 1 << 26)}
    losses, t_fwd, t_adj, rmse = [], 0.0, 0.0, []
    for k in range(steps):
        opt.zero_grad()
        img = owe_autograd.camera_film(heights(ctrl), c, hf, base_z, 2 * k * spp_step, spp_step,
                                       adjoint_pass=(2 * k + 1) * spp_step)
        t_fwd += c.last_pass_timing()[0]
        loss = ((tiles(img) - target) ** 2).mean()
        loss.backward()
        t_adj += c.last_path_adjoint_seconds()
        opt.step()
        decay.step()
        losses.append(float(loss.detach()))
        rmse.append(float(torch.sqrt((((ctrl.detach() - ct) * mask) ** 2).sum() / mask.sum())))
    res.update({"loss64_last": loss64(ctrl.detach(), 1 << 26), "loss_first": losses[0], "loss_last": losses[-1],
                "loss_mean_first10": float(np.mean(losses[:10])), "loss_mean_last10": float(np.mean(losses[-10:])),
                "forward_s_per_step": t_fwd / steps, "adjoint_s_per_step": t_adj / steps,
                "control_rmse_vs_target_first": float(torch.sqrt((ct ** 2).sum() / mask.sum())),
                "control_rmse_vs_target_last": rmse[-1],
                "control_rmse_every_20": [round(r, 7) for r in rmse[19::20]]})
    return res


def configs_study(device):
    """The other configurations' own rates: C1 (N-BK7 sphere on a floor under the sun, 256 x 256,
    one uniform wavelength per path, depth 16) in paths/s of one 64-spp pass, and C3 (the
    achromat imaging a point source onto a 1024 x 1024 detector, stochastic Fresnel branching with
    ghosts, depth 32) in walks/s over 2^24 walks."""
    import owe_cuda
    out = {}
    with owe_cuda.Context(device) as c:
        c.upload(scenes.glass_sphere_on_floor(256, 256).desc())
        c.build_bvh()
        c.set_settings(A.make_settings(seed=0, max_depth=16, rr_depth=4, wavelength_mode=A.WAVELENGTHS_UNIFORM1))
        c.run_pass(1)
        c.reset_film()
        # the configuration's own pass: 64 samples per pixel in one call, which batches 32 samples
        # of the 256 x 256 film (2^21 paths) per wavefront batch
        c.run_pass(64)
        out["c1_paths_per_s"] = 256 * 256 * 64 / c.last_pass_timing()[0]
        out["c1_pass_s"] = c.last_pass_timing()[0]
    sb, info = scenes.achromat_scene(film=1024)
    w = scenes.achromat_walk(info, seed=1, mode=A.WALK_STOCHASTIC, max_events=32)
    with owe_cuda.Context(device) as c:
        c.upload(sb.desc())
        c.build_bvh()
        c.walk(w, 0, 1 << 20)
        c.walk_reset()
        c.walk(w, 0, 1 << 24)
        out["c3_walks_per_s"] = (1 << 24) / c.walk_timing()[0]
    return out


def light_study(device, passes=8):
    """The light integrator (particles from the area light, connected to the pinhole at every
    non-specular vertex) on the bench's own scene at 1920 x 1080: particles/s over one-particle-per-
    pixel passes, and its image mean against the path integrator's on the same scene."""
    import owe_cuda
    out = {}
    with owe_cuda.Context(device) as c:
        c.upload(scenes.bvh_stress_room(WIDTH, HEIGHT).desc())
        c.build_bvh()
        means = {}
        for integrator in ("light", "path"):
            c.set_settings(A.make_settings(seed=5, max_depth=12, rr_depth=6, integrator=integrator))
            c.run_pass(1)
            c.reset_film()
            seconds = 0.0
            for _ in range(passes):
                c.run_pass(1)
                seconds += c.last_pass_timing()[0]
            means[integrator] = float(c.resolve()[0][:, :, 1].mean())
            out[f"{integrator}_per_s"] = WIDTH * HEIGHT * passes / seconds
            if integrator == "light":
                st = c.stats()
                out["light_connections_per_particle"] = st["shadow_rays"] / max(1, st["paths"])
                out["light_faults"] = st["device_faults"]
        out["mean_y_light_over_path"] = means["light"] / means["path"]
    out["unit"] = "particles/s (light), paths/s (path)"
    return out


def spawn_ranks(args):
    """`--gpus N` without a launcher: starts N copies of this script, one per GPU, with RANK,
    LOCAL_RANK, WORLD_SIZE and a loopback rendezvous set (what torch.distributed.run would set), and
    returns the first non-zero exit status (0 when all ranks succeed)."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    procs = []
    for r in range(args.gpus):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(args.gpus), LOCAL_WORLD_SIZE=str(args.gpus),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.abspath(__file__)] + sys.argv[1:], env=env))
    codes = [p.wait() for p in procs]
    return next((c for c in codes if c != 0), 0)


def run_cuda(args):
    import torch
    world, rank, local = dist_env()
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE is {world}: launch one process per GPU")
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    import owe_cuda

    desc = scenes.bvh_stress_room(WIDTH, HEIGHT).desc()
    backend = owe_cuda.CudaBackend()
    renderer = backend.create_renderer(desc, settings_for(rank), device=local)
    ctx = renderer.ctx
    info = ctx.bvh_info()
    n_pix = WIDTH * HEIGHT
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    for _ in range(max(3, args.warmup)):
        ctx.run_pass(1)

    # algorithmic traffic of a pass (counting pass, untimed)
    ctx.trace_counters(1)
    ctx.run_pass(1)
    launch_queries = ctx.trace_launch_queries()
    cnt = ctx.trace_counters(0)
    _, isec_prof, _, launches_prof = ctx.last_pass_timing()

    stats0 = ctx.stats()
    times, isec, shadow = [], [], []
    launches = 0
    gpu_index = int(os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[local]) if os.environ.get(
        "CUDA_VISIBLE_DEVICES") else local
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    with ClockSampler(gpu_index) as clocks:
        for _ in range(args.steps):
            flush.fill_(1.0)  # evict the L2 between steps
            torch.cuda.synchronize()
            ctx.run_pass(1)
            t, ti, ts, nl = ctx.last_pass_timing()
            times.append(t)
            isec.append(ti)
            shadow.append(ts)
            launches += nl
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    stats1 = ctx.stats()
    device_seconds = sum(times)
    if world > 1:
        t = torch.tensor([device_seconds], dtype=torch.float64, device=f"cuda:{local}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        device_seconds = float(t.item())
    paths_rank = stats1["paths"] - stats0["paths"]
    total_paths = paths_rank * world
    value = total_paths / device_seconds

    # end to end through the public API: a pass and the film read back to the host, every step. The
    # read-back of step k runs on a copy stream while step k + 1 renders (Renderer.resolve_async into
    # two page-locked images); every step's image has landed in host memory when the timed region
    # ends. The same loop with the synchronous resolve is timed beside it.
    e2e_steps = max(2, min(args.steps, 10))
    images = [torch.empty((HEIGHT, WIDTH, 3), dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
    for k in range(2):  # untimed: the first resolves set up their device and staging buffers
        renderer.run_pass(1)
        renderer.resolve(out=images[k])
        renderer.resolve_async(images[k])
    renderer.resolve_wait()
    torch.cuda.synchronize()
    step_settings = renderer.settings

    def e2e_loop(pipelined):
        split = []
        t0 = time.perf_counter()
        for k in range(e2e_steps):
            ta = time.perf_counter()
            # the step's inputs: the render settings (seed, depths, modes) through the public API;
            # the scene and its BVH stay resident in HBM from one step to the next
            ctx.set_settings(step_settings)
            renderer.run_pass(1)
            tb = time.perf_counter()
            if pipelined:
                renderer.resolve_async(images[k % 2])
            else:
                renderer.resolve(out=images[k % 2])
            split.append((tb - ta, time.perf_counter() - tb))
        if pipelined:
            renderer.resolve_wait()
        return time.perf_counter() - t0, split

    e2e_sync_seconds, _ = e2e_loop(False)
    e2e_seconds, split = e2e_loop(True)
    e2e_value = n_pix * world * e2e_steps / e2e_seconds
    d2h = n_pix * 3 * 8  # the resolved XYZ image (Renderer::resolve), FP64
    h2d = __import__("ctypes").sizeof(A.Settings)  # the settings record uploaded every step

    # the film over NCCL, device to device: the one exchange step of a multi-GPU render
    if world > 1:
        import distributed
        distributed.reduce_film_device(ctx)
        torch.cuda.synchronize()

    if rank == 0:
        hbm, peak_kind = peaks()
        q, nodes, prims = cnt[0], cnt[1], cnt[2]
        bytes_isec = nodes * NODE_BYTES + prims * PRIM_BYTES + q * RAY_STATE_BYTES
        # algorithmic bytes of an average launch (from the counting pass's visit counts) over the
        # average device time of the timed passes' intersect launches
        per_launch_bytes = bytes_isec / max(1, launches_prof)
        per_launch_s = sum(isec) / max(1, launches)
        achieved = per_launch_bytes / per_launch_s / 1e9
        # DRAM traffic per launch: the ncu-measured bytes per query (profiles/) times this launch's queries
        traffic = None
        try:
            with open(os.path.join(ROOT, "profiles", "kIntersect_dram_per_query.json")) as f:
                traffic = json.load(f)["dram_bytes_per_query"] * q / max(1, launches_prof)
        except (OSError, KeyError, ValueError):
            pass
        clk = clocks.summary()
        # the device's FP32 FMA rate and L2 read bandwidth, probed after the timed region
        probe = ctx.device_peaks()
        fp32_peak = probe["fp32_flops"] / 1e12
        l2_peak = probe["l2_read_bytes_per_s"] / 1e9
        flops_per_launch = (nodes * NODE_FLOPS + prims * PRIM_FLOPS) / max(1, launches_prof)
        fp32_achieved = flops_per_launch / per_launch_s / 1e12
        issue = None
        try:
            with open(os.path.join(ROOT, "profiles", "kIntersect_issue.json")) as f:
                issue = json.load(f)["issue_active"]
        except (OSError, KeyError, ValueError):
            pass
        terms = {"hbm": achieved / hbm, "l2": achieved / l2_peak, "fp32": fp32_achieved / fp32_peak}
        if issue is not None:
            terms["issue"] = issue
        bound = max(terms, key=terms.get)
        cpu_rate, cores, sample = (None, None, "skipped")
        if INTEGRATOR == "light":
            sample = "none: the reference has no CPU light integrator"
        elif not args.no_cpu_baseline:
            try:
                cpu_rate, cores, sample = cpu_reference_rate(desc)
            except BaseException as e:  # pytest.skip when the oracle was not built
                sample = f"unavailable: {e}"
        light = INTEGRATOR == "light"
        line = {
            "metric": "spectral particles/s" if light else METRIC, "value": value,
            "unit": "particles/s" if light else "paths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * device_seconds / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"mixed": "f32+f64", "fp32": "f32", "fp64": "f64"}[PRECISION], "data": "synthetic",
            "config": {"workload": workload() + (", light integrator (particles)" if light else ""),
                       "paths_per_step": n_pix, "triangles": info["triangles"],
                       "precision": {"mixed": "fp32 camera-relative + selective fp64", "fp32": "plain fp32",
                                     "fp64": "all fp64"}[PRECISION], "l2": "flushed between steps (512 MB write)",
                       "parallelism": f"replicated scene, dp{world} over sample streams"},
            "gpu_launches": None,
            "rays_per_s": (stats1["segments"] - stats0["segments"] + stats1["shadow_rays"] - stats0["shadow_rays"])
                          * world / device_seconds,
            "segments_per_path": (stats1["segments"] - stats0["segments"]) / max(1, paths_rank),
            "wall_seconds": wall,
            "intersect_share": sum(isec) / sum(times),
            "shadow_share": sum(shadow) / sum(times),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_kind": peak_kind, "traffic": traffic, "kernel": "kIntersect",
                         "binding_term": bound,
                         "terms": {k: round(v, 4) for k, v in terms.items()},
                         "term_sources": {"hbm": f"algorithmic bytes / launch time vs {peak_kind} copy bandwidth",
                                          "l2": f"the same bytes vs the probed L2 read bandwidth ({l2_peak:.0f} GB/s)",
                                          "fp32": f"{NODE_FLOPS} flops per node visit + {PRIM_FLOPS} per primitive test "
                                                  f"vs the probed FP32 FMA rate ({fp32_peak:.1f} TFLOP/s)",
                                          "issue": "ncu issue-active fraction of the kernel (profiles/kIntersect_issue.json)"},
                         "fp32_tflops": fp32_achieved, "fp64_peak_tflops": probe["fp64_flops"] / 1e12,
                         "bytes_per_launch": per_launch_bytes,
                         "per_query": {"nodes": nodes / max(1, q), "prims": prims / max(1, q)},
                         "queries_per_pass": q, "launches_per_pass": launches_prof,
                         "queries_per_launch": launch_queries},
            "clocks": clk,
            "cpu_baseline": {"value": cpu_rate, "unit": "particles/s" if light else "paths/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": e2e_value, "unit": "particles/s" if light else "paths/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "value_at_median_step": n_pix * world / statistics.median(a + b for a, b in split),
                    "steps": e2e_steps, "pass_ms": [round(1e3 * a, 2) for a, _ in split],
                    "resolve_ms": [round(1e3 * b, 2) for _, b in split],
                    "value_synchronous_resolve": n_pix * world * e2e_steps / e2e_sync_seconds,
                    "note": "per step through owe_cuda.Renderer: the settings record set, one pass, the resolved image read back into pinned host memory (resolve_async: the copy of step k overlaps the pass of step k + 1; all copies have landed when the timed region ends; value_synchronous_resolve waits for each copy); the scene and BVH are uploaded once and stay resident in HBM"},
            "faults": stats1["device_faults"],
        }
        if not args.no_extras and world == 1 and not light:
            line["precision_study"] = precision_study(local)
            line["adjoint_study"] = adjoint_study(local)
            line["configs_study"] = configs_study(local)
            line["light_study"] = light_study(local)
        # our own kernel launches in the timed region: intersect, medium, two surface kernels, the
        # shadow visibility and its contributions per bounce, and generate + film per step; for
        # particles intersect, event, visibility and splats per bounce, and emit with the emitters'
        # own connections (visibility and splats) per step
        line["gpu_launches"] = int(4 * launches + 3 * args.steps) if light else int(6 * launches + 2 * args.steps)
        print(json.dumps(line))
    renderer.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the RMSE-at-equal-paths precision study and the adjoint/forward study")
    ap.add_argument("--width", type=int, default=1920, help="film width (a smaller case for profiling)")
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--precision", default="mixed", choices=sorted(PRECISIONS),
                    help="mixed: FP32 camera-relative + selective FP64 (the product); fp64: the all-FP64 "
                         "instantiation of the same kernels it is compared with")
    ap.add_argument("--c5", type=int, default=-1, metavar="STEPS",
                    help="run only the large-adjoint study (caustic room at 1920x1080, depth 24) with STEPS "
                         "gradient steps (0: timing and memory alone) and print its JSON")
    ap.add_argument("--c5-spp", type=int, default=1024,
                    help="samples per pixel of the large-adjoint study's timed forward pass and adjoint")
    ap.add_argument("--c5-step-spp", type=int, default=8, help="samples per pixel of each optimisation step")
    ap.add_argument("--integrator", default="path", choices=["path", "light"],
                    help="path: the headline camera-path integrator; light: particles from the emitters, "
                         "measured in particles/s on the same scene")
    args = ap.parse_args()
    globals()["WIDTH"], globals()["HEIGHT"] = args.width, args.height
    globals()["PRECISION"] = args.precision
    globals()["INTEGRATOR"] = args.integrator
    if args.impl == "reference":
        return run_reference(args)
    if args.c5 >= 0:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"c5_study": c5_study(0, spp_timing=args.c5_spp, steps=args.c5, spp_step=args.c5_step_spp)}))
        return 0
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return spawn_ranks(args)
    return run_cuda(args)


if __name__ == "__main__":
    sys.exit(main())
