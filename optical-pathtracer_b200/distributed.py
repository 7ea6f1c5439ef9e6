"""Rendering one image on several GPUs: one process per GPU, the sample streams of a render split
into contiguous blocks across the ranks, and one exchange, the film (and, for the adjoints, one
all-reduce of the height gradient).

A render of S samples per pixel draws the streams (hashCombine(seed, pixel), 0 .. S - 1) (the pass
index of CpuRenderer::pass, src/owe/backends/cpu/cpu_backend.cpp:66). Rank r of W renders the
block stream_block(S, W, r) on its own device, with the scene and BVH replicated; the ranks then
add their films' compensated XYZ sums and sample counts with one all-reduce (NCCL over NVLink on
GPUs, gloo on CPU) and divide. The ranks together draw exactly the streams one device would, so
the result equals the one-device film up to the order of the final additions.
"""
import numpy as np


def stream_block(total, world, rank):
    """(first stream, count) of rank `rank` of `world` for `total` samples per pixel: contiguous,
    sizes differing by at most one, in rank order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    if total < 0:
        raise ValueError("negative sample count")
    base, extra = divmod(total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def reduce_film(sums, samples, group=None):
    """All-reduce of the films' XYZ sums and sample counts (float64, in place on copies); every rank
    gets the totals."""
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    device = f"cuda:{torch.cuda.current_device()}" if backend == "nccl" else "cpu"
    t = torch.from_numpy(np.concatenate([np.ascontiguousarray(sums, np.float64).ravel(),
                                         np.ascontiguousarray(samples, np.float64).ravel()])).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    t = t.cpu().numpy()
    n = np.size(sums)
    return t[:n].reshape(np.shape(sums)), t[n:].reshape(np.shape(samples))


def reduce_film_device(ctx, group=None):
    """The film's sums and sample counts all-reduced where they live: read into CUDA tensors on the
    context's device (owec_read_film_device) and summed there over NCCL (NVLink between the GPUs).
    Returns (sums (height, width, 3), samples (height, width)) as CUDA tensors, the same on every rank."""
    import torch
    import torch.distributed as dist
    n = ctx.width * ctx.height
    dev = f"cuda:{torch.cuda.current_device()}"
    buf = torch.empty(4 * n, dtype=torch.float64, device=dev)
    ctx.read_film_device(buf.data_ptr(), buf.data_ptr() + 3 * n * 8)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    return buf[:3 * n].view(ctx.height, ctx.width, 3), buf[3 * n:].view(ctx.height, ctx.width)


def render(ctx, total_spp, group=None, spp_per_pass=None):
    """Renders rank's share of `total_spp` samples per pixel with `ctx` (an owe_cuda.Context with its
    scene, BVH and settings in place, film reset), reduces the films over `group` and returns the
    per-pixel mean XYZ (height, width, 3), the same on every rank."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    first, count = stream_block(total_spp, world, rank)
    ctx.set_pass_index(first)
    step = count if spp_per_pass is None else max(1, int(spp_per_pass))
    done = 0
    while done < count:
        n = min(step, count - done)
        ctx.run_pass(n)
        done += n
    if dist.get_backend(group) == "nccl":
        sums, samples = (t.cpu().numpy() for t in reduce_film_device(ctx, group))
    else:
        sums, samples = ctx.read_film()
        sums, samples = reduce_film(sums, samples, group)
    with np.errstate(invalid="ignore", divide="ignore"):
        mean = np.where(samples[..., None] > 0, sums / np.maximum(samples, 1)[..., None], 0.0)
    return mean


def _all_reduce_host(values, group):
    """Sum of a float64 host array over the ranks (on the GPU under NCCL, on the CPU under gloo)."""
    import torch
    import torch.distributed as dist
    device = f"cuda:{torch.cuda.current_device()}" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(np.ascontiguousarray(values, np.float64)).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def walk_gradient(ctx, desc, total_walks, g, group=None):
    """The gradient of sum_b g_b bins_b over walks 0 .. total_walks - 1 with respect to the heights,
    shared out over the ranks: rank r replays its contiguous block of walks (owec_walk_adjoint
    normalises the film by the walks of its own call, so each rank's gradient is weighted by its
    share), then one all-reduce of dLoss/dHeights. Every rank gets the whole gradient."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    first, count = stream_block(total_walks, world, rank)
    part = ctx.walk_adjoint(desc, first, count, g) * (count / total_walks) if count else None
    if part is None:
        part = np.zeros(getattr(ctx, "_hf_n", 0))
    return _all_reduce_host(part, group)


def path_gradient(ctx, total_spp, g, group=None, first_pass=0):
    """The gradient of sum_p g_p . film_p for the film of samples first_pass .. first_pass +
    total_spp - 1 with respect to the heights, shared out over the ranks by sample streams as
    render() shares the film: rank r replays its block (owec_path_adjoint, which normalises by its
    own samples per pixel, so each rank's gradient is weighted by its share), then one all-reduce of
    dLoss/dHeights."""
    import torch.distributed as dist
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    first, count = stream_block(total_spp, world, rank)
    part = ctx.path_adjoint(first_pass + first, count, g) * (count / total_spp) if count else None
    if part is None:
        part = np.zeros(getattr(ctx, "_hf_n", 0))
    return _all_reduce_host(part, group)
