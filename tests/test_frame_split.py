"""One frame split across ranks, on the CPU.

rc_frame_part_range (host arithmetic behind the C ABI) must tile the frame:
parts in order cover SPPM iterations [0, it) and samples [0, spp) without
gaps or overlaps, each part's samples being whole iteration blocks of
rc_render_frame.  The world-size-2 test runs the split as bench.py and
retrocam_b200/frame_split.py run it -- a part per rank, then one sum of the
accumulation and variance images onto rank 0 -- with the oracle rendering
each part and the sum over gloo, and compares rank 0's images and
denoised frame with one process rendering the whole frame: the G-buffer and
albedo (written by the part holding sample 0) bit for bit, the sums within
the tolerance of a different float addition order.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import REPO


@pytest.mark.parametrize("spp,iters", [(1, 0), (5, 0), (16, 0), (128, 16), (16, 16), (7, 3), (12, 1)])
@pytest.mark.parametrize("parts", [1, 2, 3, 4, 8])
def test_part_ranges_tile_the_frame(product, spp, iters, parts):
    s_next, k_next = 0, 0
    for p in range(parts):
        k0, k1, s0, s1 = product.frame_part_range(spp, iters, p, parts)
        assert s0 == s_next and s1 >= s0
        if iters:
            assert k0 == k_next and k1 >= k0
            # whole iteration blocks: rc_render_frame's block k is [k*spp/it, (k+1)*spp/it)
            assert s0 == k0 * spp // iters and s1 == k1 * spp // iters
            k_next = k1
        else:
            assert k0 == k1 == 0
        s_next = s1
    assert s_next == spp and k_next == iters


def test_part_range_rejects_bad_arguments(product):
    for args in ((0, 0, 0, 1), (4, 5, 0, 1), (4, 2, 2, 2), (4, 2, -1, 2), (4, 2, 0, 0)):
        with pytest.raises(product.RetroCamError):
            product.frame_part_range(*args)


WORKER = r"""
import os, sys
sys.path.insert(0, {repo!r}); sys.path.insert(0, os.path.join({repo!r}, "oracle"))
import numpy as np, torch, torch.distributed as dist
import pyoracle as po
from retrocam_b200 import api, scenes
dist.init_process_group("gloo")
rank, world = dist.get_rank(), dist.get_world_size()
orc, _ = po.load(build=False)
w = scenes.export_frame()
sc = scenes.build_scene(w.scene, orc, po.MAT)
cam = scenes.camera(w.orbit, w.lens, orc)
W, H, spp, iters, N, hs, r0, alpha = 48, 32, 6, 3, 20000, 1 << 16, 0.02, 0.7

def part(p, parts):
    # rc_render_frame_part restated over the oracle: radius advanced to k0,
    # then per iteration trace -> render the block -> gather -> shrink
    k0, k1, s0, s1 = api.frame_part_range(spp, iters, p, parts)
    bufs = po.alloc_images(W, H)
    r = np.float32(r0)
    for k in range(k0):
        r = orc.lib.or_sppm_next_radius(r, k, alpha)
    for k in range(k0, k1):
        b0, b1 = k * spp // iters, (k + 1) * spp // iters
        ph, hd, nx, cnt, _ = orc.photon_trace(sc, N, r, k * 7919 + 6271, hs)
        orc.render(sc, cam, (1, 1.0), W, H, b0, b1 - b0, buffers=bufs)
        orc.photon_gather(sc, cam, W, H, r, hs, ph, hd, nx, bufs[0], weight=float(b1 - b0))
        r = orc.lib.or_sppm_next_radius(r, k, alpha)
    return bufs

bufs = part(rank, world)
acc, var = torch.from_numpy(bufs[0]), torch.from_numpy(bufs[3])
dist.reduce(acc, dst=0)
dist.reduce(var, dst=0)
if rank == 0:
    whole = part(0, 1)
    np.savez({out!r}, acc=acc.numpy(), var=var.numpy(), gb=bufs[1], ga=bufs[2], w_acc=whole[0], w_var=whole[3],
             w_gb=whole[1], w_ga=whole[2])
dist.destroy_process_group()
print("DONE", rank, flush=True)
"""


def test_split_frame_over_gloo_matches_one_process(tmp_path, oracle_libs, product):
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    out = str(tmp_path / "split.npz")
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), OMP_NUM_THREADS="2")
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER.format(repo=REPO, out=out)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    logs = [p.communicate(timeout=600)[0] for p in procs]
    for p, log in zip(procs, logs):
        assert p.returncode == 0, log[-3000:]
    r = np.load(out)
    # the G-buffer and albedo come from the part holding sample 0: exact
    assert np.array_equal(r["gb"], r["w_gb"]) and np.array_equal(r["ga"], r["w_ga"])
    # sums of the same terms in another order; sample counts exact
    np.testing.assert_array_equal(r["acc"][..., 3], r["w_acc"][..., 3])
    np.testing.assert_allclose(r["acc"], r["w_acc"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(r["var"], r["w_var"], rtol=1e-5, atol=1e-6)
    assert np.abs(r["w_acc"][..., :3]).max() > 0
    # the denoised frames: the colour edge-stopping weight exp(-dL^2 / (var +
    # 1e-6)) amplifies last-bit input differences where the variance is
    # tiny, so a few elements differ by up to ~2e-4 relative; the image mean
    # agrees to 1e-6
    import pyoracle as po
    orc = oracle_libs[0]
    p = po.AtrousParams(1, 5, 1.0, 128.0, 1.0, 0, 1.0)
    a = orc.denoise(r["acc"], r["gb"], r["ga"], r["var"], 48, 32, 6, p)
    b = orc.denoise(r["w_acc"], r["w_gb"], r["w_ga"], r["w_var"], 48, 32, 6, p)
    np.testing.assert_allclose(a, b, rtol=1e-3, atol=1e-4)
    assert abs(a.mean() - b.mean()) <= 1e-6 * abs(b.mean())
