"""Several images in one batched fit (each image keeps its own tiles, file and RD score).

Tiles of every image are concatenated into ONE ``BatchedFit`` (one scoring launch per tile-size
class per round for the whole batch) or one ``RefinedFit``; a per-image tile range maps the
results back.  Tiles never interact, so a batched fit selects exactly what per-image fits select.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import candidates, quadtree
from .synth import srgb_u8_to_linear


@dataclass
class ImageTiles:
    """One image of a batch: linear pixels, quadtree tiles, tile patches, candidate records."""

    image: np.ndarray
    tiles: list
    patches: list
    pools: list  # packed candidate records (numpy PRIM_DTYPE) per tile

    @property
    def size(self) -> tuple[int, int]:
        return self.image.shape[1], self.image.shape[0]


def _cands(args):
    patch, q = args
    from .fit import pack_cands

    return pack_cands(candidates.tile_candidates(patch, q))


def prepare_image(u8: np.ndarray, quality: int = 75, executor=None, threshold: float = 100.0,
                  pools: bool = True) -> ImageTiles:
    """Quadtree (8-64 px, split while u8 luminance variance > ``threshold``), tiles and the
    reference's candidate pools (host; ``executor`` maps over tiles when given; ``pools=False``
    skips them, for fits whose pools are generated on the device)."""
    img = srgb_u8_to_linear(u8)
    tiles = quadtree.decompose(img, rule="variance", threshold=threshold, min_tile=8, max_tile=64, image_u8=u8)
    patches = quadtree.extract_tiles(img, tiles, 64)
    recs = None
    if pools:
        jobs = [(p, quality) for p in patches]
        recs = list(executor.map(_cands, jobs, chunksize=32)) if executor is not None else [_cands(j) for j in jobs]
    return ImageTiles(img, tiles, patches, recs)


class ImageBatch:
    """Images whose tiles are fitted together."""

    def __init__(self, images: list[ImageTiles], quality: int = 75, cap: int = 16, device: int = 0):
        self.images = images
        self.quality = quality
        self.cap = cap
        self.device = device
        counts = [len(im.tiles) for im in images]
        self.tile_off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        self.patches = [p for im in images for p in im.patches]
        self.pools = [p for im in images for p in im.pools] if all(im.pools is not None for im in images) else None

    @property
    def n_pixels(self) -> int:
        return int(sum(p.shape[0] ** 2 for p in self.patches))

    def arrays(self, kinds=None):
        """Flat host inputs of ``BatchedFit.from_arrays`` (optionally only candidate ``kinds``)."""
        pools = self.pools if kinds is None else [p[np.isin(p["kind"], kinds)] for p in self.pools]
        pixels = np.concatenate([p.reshape(-1, 3) for p in self.patches])
        sizes = np.array([p.shape[0] for p in self.patches], np.int32)
        return pixels, sizes, np.concatenate(pools), np.array([len(p) for p in pools], np.int64)

    def plain_fit(self, autotune: bool = True):
        from .fit import BatchedFit

        pixels, sizes, recs, cnt = self.arrays()
        fit = BatchedFit.from_arrays(pixels, sizes, recs, cnt, self.quality, caps=[self.cap] * len(sizes),
                                     device=self.device)
        if autotune:
            fit.autotune()
        return fit

    def refined_fit(self, steps: int = 10, lr: float = 1e-2, kinds=(0, 1), autotune: bool = True,
                    use_graph: bool = True, residual: bool = False):
        from .fit import BatchedFit
        from .refine import RefinedFit

        pixels, sizes, recs, cnt = self.arrays(kinds)
        fit = BatchedFit.from_arrays(pixels, sizes, recs, cnt, self.quality, caps=[self.cap] * len(sizes),
                                     device=self.device, reserve=0)
        fit.use_closed_form_init(True)
        if autotune:
            fit.autotune()
        return RefinedFit(fit, steps=steps, lr=lr, use_graph=use_graph, residual=residual)

    def refined_fit_device(self, steps: int = 100, lr: float = 1e-2, autotune: bool = True, use_graph: bool = True):
        """The refined fit with its constant + linear pools generated on the device for every tile of
        every image (``pools.DeviceRefinedFit``): generation, init round, ``steps`` Adam steps and the
        wire-grid snap in one CUDA graph; only the tile pixels go to the device."""
        import torch

        from .pools import DeviceRefinedFit

        pixels, sizes = self.tile_pixels()
        dev = torch.device("cuda", self.device)
        src4 = torch.zeros((len(pixels), 4), dtype=torch.float32, device=dev)
        src4[:, :3] = torch.from_numpy(pixels).to(dev)
        return DeviceRefinedFit(src4, sizes, self.quality, caps=[self.cap] * len(sizes), steps=steps, lr=lr,
                                use_graph=use_graph, autotune=autotune)

    def tile_pixels(self):
        """Tile pixels of the whole batch, tile-major (float32 (n, 3)), and the tile sides."""
        pixels = np.concatenate([p.reshape(-1, 3) for p in self.patches])
        return pixels, np.array([p.shape[0] for p in self.patches], np.int32)

    def image_stacks(self, stacks: list) -> list[list]:
        """Split per-tile stacks of the whole batch into per-image lists."""
        return [stacks[self.tile_off[i]:self.tile_off[i + 1]] for i in range(len(self.images))]

    def rd_per_image(self, stacks: list) -> list[dict]:
        """RD of every image's file: its tiles' stacks (quantised primitives as given), RES0/RES1
        from their render, written as a WEFT file and decoded."""
        from . import render
        from .encode import encode_fit, rd_score

        out = []
        for im, st in zip(self.images, self.image_stacks(stacks)):
            w, h = im.size

            class _R:
                def __init__(self, p):
                    self.primitives = p
                    self.residual_rgb = (0, 0, 0)

            pw, ph = ((w + 63) // 64) * 64, ((h + 63) // 64) * 64
            full = render.render_scene_adaptive([_R(s) for s in st], im.tiles, pw, ph)
            recon = [full[t.y:t.y + t.size, t.x:t.x + t.size] for t in im.tiles]
            blob = encode_fit(w, h, self.quality, im.tiles, im.patches, st, recon)
            out.append(rd_score(im.image, blob, self.quality))
        return out
