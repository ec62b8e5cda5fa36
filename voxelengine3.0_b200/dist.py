"""Multi-GPU plumbing: one process per GPU.

Replica mode (the default): frames, views and requests are independent;
every rank holds its own copy of the octree and its own radiance cache and
renders its share of the work.  The only communication is for measurement: a
barrier around the timed region and the max (time) / sum (rays) over ranks.

Split frames (SplitFrame): one frame of one view too large for one GPU.
Each rank renders a band of rows; the frame's cache deposits are exchanged
once (an all-gather of each rank's records, NCCL over NVLink) and merged by
every rank in rank order, so all ranks' caches stay identical; each rank
then runs the AvgPass of its band and the bands are gathered.
"""
from __future__ import annotations

import dataclasses
import datetime
import os
from typing import Dict, Iterable, List, Optional, Sequence, Tuple


def env_rank() -> tuple:
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 300.0, device: Optional[int] = None):
    """Initialises torch.distributed when WORLD_SIZE > 1; returns the module or None."""
    rank, world, local = env_rank()
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist

    if backend == "nccl":
        torch.cuda.set_device(local if device is None else device)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def frame_assignment(n_steps: int, rank: int, world: int, period: int) -> List[int]:
    """Orbit frames of one rank: rank r renders frames r, r+world, r+2*world,
    ... (mod the orbit period) — equal work per rank (weak scaling)."""
    return [(rank + world * i) % period for i in range(n_steps)]


def split_evenly(items: Sequence, rank: int, world: int) -> list:
    """Contiguous near-equal shares of a work list (views or requests)."""
    n = len(items)
    lo = n * rank // world
    hi = n * (rank + 1) // world
    return list(items[lo:hi])


def _reduce(value: float, dist, op, device=None) -> float:
    if dist is None:
        return float(value)
    import torch

    backend = dist.get_backend()
    dev = device if device is not None else ("cuda" if backend == "nccl" else "cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value: float, dist=None, device=None) -> float:
    if dist is None:
        return float(value)
    return _reduce(value, dist, dist.ReduceOp.MAX, device)


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    if dist is None:
        return float(value)
    return _reduce(value, dist, dist.ReduceOp.SUM, device)


def barrier(dist=None) -> None:
    if dist is not None:
        dist.barrier()


def shutdown(dist=None) -> None:
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# split frames
# ---------------------------------------------------------------------------
def band_rows(height: int, rank: int, world: int) -> Tuple[int, int]:
    """Rows [lo, hi) of one rank's band: contiguous, near-equal, in rank order."""
    if height < world:
        raise ValueError(f"a frame of {height} rows cannot be split across {world} ranks")
    return height * rank // world, height * (rank + 1) // world


_IMAGE_OUTPUTS = ("voxel_id", "hit_node", "rgb", "mapped", "mapped8")
_RENDER_OUTPUTS = ("gbuffer", "path_rgb")
_RECORD_WORDS = 8  # ve_split_record: 8 x 32-bit words


class SplitFrame:
    """Renders frames of one view across the ranks of a process group.

    `renderer` is a ve_b200.Renderer (or an object with its render /
    split_export / split_merge / split_resolve methods); `dist` the
    torch.distributed module after init_process_group, or None for one rank.
    Record exchange and row gathers run on `device` ("cuda" under NCCL).
    """

    def __init__(self, renderer, scene_id: int, dist=None, device=None):
        import torch

        self.r = renderer
        self.scene_id = scene_id
        self.dist = dist
        self.rank = dist.get_rank() if dist is not None else 0
        self.world = dist.get_world_size() if dist is not None else 1
        if device is None:
            device = "cuda" if dist is None or dist.get_backend() == "nccl" else "cpu"
        self.device = torch.device(device)
        self._buf = None
        self._images: Dict[str, object] = {}  # pinned host images, reused frame to frame
        self.last: Dict[str, object] = {}

    def _image(self, name: str, fc):
        """A pinned full-size host image for output `name`."""
        import numpy as np
        import torch

        shape = {"voxel_id": (fc.height, fc.width), "hit_node": (fc.height, fc.width),
                 "rgb": (fc.height, fc.width, 3), "mapped": (fc.height, fc.width, 3),
                 "mapped8": (fc.height, fc.width, 4)}[name]
        dtype = {"voxel_id": np.uint32, "hit_node": np.uint32, "mapped8": np.uint8}.get(name, np.float32)
        tdtype = {np.uint32: torch.int32, np.uint8: torch.uint8, np.float32: torch.float32}[dtype]
        t = self._images.get(name)
        if t is None or tuple(t.shape) != shape:
            t = torch.empty(shape, dtype=tdtype, pin_memory=torch.cuda.is_available())
            self._images[name] = t
        return t.numpy().view(dtype)

    def _records(self, cap: int):
        import torch

        need = max(cap, 1) * _RECORD_WORDS
        if self._buf is None or self._buf.numel() < need:
            self._buf = torch.empty(need, dtype=torch.int32, device=self.device)
        return self._buf

    def _sync(self) -> None:
        import torch

        if self.device.type == "cuda":
            torch.cuda.current_stream(self.device).synchronize()

    def exchange(self, local, n: int):
        """All-gathers every rank's first records of `local` (n of them here):
        returns (parts, counts, stride) with part k at record k * stride."""
        import torch

        if self.dist is None:
            return local, [int(n)], max(int(n), 1)
        t = torch.tensor([int(n)], dtype=torch.int64, device=self.device)
        counts_t = [torch.zeros_like(t) for _ in range(self.world)]
        self.dist.all_gather(counts_t, t)
        counts = [int(c.item()) for c in counts_t]
        stride = max(max(counts), 1)
        mine = local[: stride * _RECORD_WORDS]
        if self.dist.get_backend() == "nccl":
            parts = torch.empty(self.world * stride * _RECORD_WORDS, dtype=torch.int32, device=self.device)
            self.dist.all_gather_into_tensor(parts, mine)
        else:
            lst = [torch.empty_like(mine) for _ in range(self.world)]
            self.dist.all_gather(lst, mine)
            parts = torch.cat(lst)
        self._sync()  # the renderer's stream reads the parts next
        return parts, counts, stride

    def gather_rows(self, image, lo: int, hi: int, height: int):
        """Full image from every rank's band [lo, hi) of a (height, ...) array."""
        import numpy as np
        import torch

        if self.dist is None:
            return image
        if image.dtype == np.uint8 and image.shape[-1] == 4:  # RGBA8: one 32-bit element per pixel
            flat = np.ascontiguousarray(image).view(np.uint32)[..., 0]
            return self.gather_rows(flat, lo, hi, height).view(np.uint8).reshape(image.shape)
        rows = max(height * (k + 1) // self.world - height * k // self.world for k in range(self.world))
        band = np.zeros((rows,) + image.shape[1:], image.dtype)
        band[: hi - lo] = image[lo:hi]
        if band.dtype.itemsize != 4:
            raise ValueError("rows of 32-bit elements only")
        t = torch.from_numpy(band.view(np.int32)).to(self.device)
        lst = [torch.empty_like(t) for _ in range(self.world)]
        self.dist.all_gather(lst, t)
        out = np.empty_like(image)
        for k, part in enumerate(lst):
            a, b = band_rows(height, k, self.world)
            out[a:b] = part.cpu().numpy().view(image.dtype)[: b - a]
        return out

    def render(self, camera, fc, outputs: Iterable[str] = ("rgb",), gather: bool = True) -> Dict[str, object]:
        """One frame; returns full-size host images (only this rank's band
        rows are filled when gather=False).  Without a gather (or on one
        rank) the images are pinned buffers that the next call reuses."""
        from . import FRAME_SPLIT

        want = list(outputs)
        lo, hi = band_rows(fc.height, self.rank, self.world)
        f = dataclasses.replace(fc, flags=fc.flags | FRAME_SPLIT, row_begin=lo, row_end=hi)
        out = dict(self.r.render(self.scene_id, camera, f, outputs=[k for k in want if k in _RENDER_OUTPUTS]))
        # a band's deposits land on its pixels' primary voxels: at most one
        # record per pixel of the largest band
        cap = max(fc.height * (k + 1) // self.world - fc.height * k // self.world for k in range(self.world)) * fc.width
        buf = self._records(cap)
        n = self.r.split_export(self.scene_id, buf, cap)
        parts, counts, stride = self.exchange(buf, n)
        dropped = self.r.split_merge(self.scene_id, parts, counts, stride)
        images = {k: self._image(k, fc) for k in want if k in _IMAGE_OUTPUTS}
        if hasattr(self.r, "split_resolve_into"):
            self.r.split_resolve_into(self.scene_id, camera, f, images)
            out.update(images)
        else:
            out.update(self.r.split_resolve(self.scene_id, camera, f, list(images)))
        if gather:
            for k in list(out):
                a = out[k]
                if k == "path_rgb":  # pixel-major: rows of width * spp paths
                    a = a.reshape(fc.height, fc.width * fc.spp, 3)
                    out[k] = self.gather_rows(a, lo, hi, fc.height).reshape(-1, 3)
                else:
                    out[k] = self.gather_rows(a, lo, hi, fc.height)
        self.last = {"band": (lo, hi), "records": n, "counts": counts, "dropped": dropped}
        return out
