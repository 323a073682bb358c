"""One export frame split across GPUs (one process per GPU).

Each rank renders its contiguous share of the frame's SPPM iterations and
their sample blocks with rc_render_frame_part (seeds are frame indices and
iteration numbers, so the parts together render exactly the samples and
photon maps of rc_render_frame), then the partial accumulation (RGBA32F:
radiance sums and sample counts) and variance (R32F: sums of luma^2) images
are summed onto the root rank with one collective each -- 20 bytes per pixel,
8.2 MB at 854x480 -- and the root, whose part holds sample 0 and so the
G-buffer and albedo, sets the frame's sample count and denoises.  This is the
only exchange the path has.  The collectives run on the context's own
stream (a torch stream), in place on the context's device images.

The sum differs from the one-device frame only in the order of the float
additions (part sums added together instead of one running sum).
"""
from __future__ import annotations

from . import api


class _DeviceArray:
    """A device buffer described by __cuda_array_interface__ (version 3), so
    torch can view the context's images without copying them."""

    def __init__(self, ptr: int, shape: tuple, typestr: str):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False), "version": 3,
                                         "strides": None}


def image_tensors(ctx: api.Context, device):
    """torch views (no copy) of the context's accum (H, W, 4) float32 and
    variance (H, W) float32 images on `device`."""
    import torch
    p = ctx.image_pointers()
    H, W = ctx.height, ctx.width
    acc = torch.as_tensor(_DeviceArray(p["accum"], (H, W, 4), "<f4"), device=device)
    var = torch.as_tensor(_DeviceArray(p["variance"], (H, W), "<f4"), device=device)
    return acc, var


def render_frame_split(ctx: api.Context, dist, stream, cam, settings, spp, sppm, r0, sppm_iters, atrous,
                       root: int = 0, denoise: bool = True):
    """rc_render_frame's frame over the ranks of `dist` (torch.distributed,
    NCCL): this rank's part, the sum of every part's accumulation and
    variance on `root`, and there the sample count and the denoise.  `ctx`
    must run on `stream` (Context.set_stream(stream.cuda_stream)): the
    collectives are issued on it after the part's kernels."""
    import torch
    rank, world = dist.get_rank(), dist.get_world_size()
    ctx.render_frame_part(cam, settings, spp, sppm, r0, sppm_iters, rank, world)
    if world > 1:
        acc, var = image_tensors(ctx, stream.device)
        with torch.cuda.stream(stream):
            dist.reduce(acc, dst=root)
            dist.reduce(var, dst=root)
    if rank == root:
        ctx.set_total_samples(spp)
        if denoise:
            ctx.denoise(atrous, read=False)
