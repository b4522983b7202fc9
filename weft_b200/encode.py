"""From fitted stacks to a WEFT file and its RD score (host side, GPU render).

``encode_fit`` mirrors the reference's build phase for the primitive-stack
basis (src/weft/encoder.py:2986-3005, :3248-3372): per tile RES0 = the
rounded mean error of the fitted render (x255, clipped to +-127) and RES1 = the
4x4 block means of the remaining error (same quantization); the container is
written by ``weft_b200.bitstream``.  ``decode_file`` parses a file and renders
it with the GPU decoder walk; ``rd_score`` is PSNR - lambda_rd * BPP of the
decoded file (src/weft/encoder.py:3926-3931, :4008-4011).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import bitstream, rate, render
from .candidates import Cand


@dataclass
class _Rec:
    primitives: list
    residual_rgb: tuple = (0, 0, 0)


def residuals_from_recon(patches, recon):
    """RES0 ints and RES1 int8 grids per tile from source patches and the fitted
    render (clipped composite, no residuals), as the reference's build phase."""
    res0, res1 = [], []
    for p, r in zip(patches, recon):
        bias = (p - r).mean(axis=(0, 1))
        rgb = tuple(int(np.clip(np.round(float(b) * 255.0), -127, 127)) for b in bias)
        res0.append(rgb)
        pred2 = np.clip(r + np.array(rgb, np.float32)[None, None, :] / 255.0, 0.0, 1.0)
        err = p - pred2
        ts = p.shape[0]
        s = ts // 4
        grid = err.reshape(4, s, 4, s, 3).mean(axis=(1, 3))
        res1.append(np.clip(np.round(grid * 255.0), -127.0, 127.0).astype(np.int8))
    return res0, res1


def residuals_from_fit_gpu(fit):
    """RES0 and RES1 of a ``BatchedFit``'s current selection, built on the GPU from its resident
    tile pixels and composite (``weftk_build_residuals``); the same bytes as
    ``residuals_from_recon(patches, fit.recon_tiles())``."""
    import torch

    from . import _lib

    d = fit.device
    r0 = torch.zeros((fit.n, 3), dtype=torch.int8, device=d)
    r1 = torch.zeros((fit.n, 4, 4, 3), dtype=torch.int8, device=d)
    _lib.check(fit.lib.weftk_build_residuals(_lib.ptr(fit.t_src), _lib.ptr(fit.t_bg), 1, _lib.ptr(fit.t_px_off),
                                             _lib.ptr(fit.t_size), fit.n, _lib.ptr(r0), _lib.ptr(r1),
                                             torch.cuda.current_stream(d).cuda_stream), "weftk_build_residuals")
    res0 = [tuple(int(v) for v in row) for row in r0.cpu().numpy()]
    return res0, list(r1.cpu().numpy())


def encode_fit(width, height, quality, tiles, patches, stacks, recon, with_res0=True, with_res1=True):
    """File bytes for fitted ``stacks`` (per-tile primitives) whose clipped renders are ``recon``."""
    res0, res1 = residuals_from_recon(patches, recon)
    return bitstream.encode_weft(width, height, quality, tiles, stacks,
                                 residuals=res0 if with_res0 else None, res1_maps=res1 if with_res1 else None)


def decode_file(blob: bytes, target_width=None, target_height=None) -> np.ndarray:
    """Decode a primitive-stack WEFT file with the GPU decoder walk (linear float32 RGB); the target
    defaults to the file's width and height.  A file with a DCT residual block takes the raster
    branch: walk at the encoded size, DCT residual, u8 BILINEAR resize to the target."""
    wf = bitstream.decode_weft(blob)
    tiles = [type("QT", (), {"x": x, "y": y, "size": s})() for x, y, s in wf.qtree]
    stacks = bitstream.decode_tiles(wf.prim_raw, wf.toc)
    recs = []
    for i, st in enumerate(stacks):
        prims = [Cand(k, g, c0, c1, a) for k, g, c0, c1, a in st]
        recs.append(_Rec(prims, tuple(wf.residuals[i]) if wf.residuals is not None else (0, 0, 0)))
    maps = [m.astype(np.float32) / 255.0 for m in wf.res1_maps] if wf.res1_maps is not None else None
    ew = int(wf.meta.get("encode_width", wf.width))
    eh = int(wf.meta.get("encode_height", wf.height))
    tw, th = int(target_width or wf.width), int(target_height or wf.height)
    if wf.dct_payload is None:
        return render.render_scene_adaptive(recs, tiles, ew, eh, maps, 4, tw, th)
    # raster branch (src/weft/decoder.py:446-518): walk at the encoded size, add the DCT
    # residual, then u8 + BILINEAR resize when the target differs
    from . import raster

    img = render.render_scene_device(recs, tiles, ew, eh, maps)
    img = raster.apply_dct(img, wf.dct_payload, wf.qtree)
    return raster.resize(img, tw, th).cpu().numpy()


def rd_score(image: np.ndarray, blob: bytes, quality: int) -> dict:
    """RD score of a file against the linear source image."""
    h, w = image.shape[:2]
    dec = decode_file(blob)
    p = rate.psnr(image, dec)
    bpp = len(blob) * 8.0 / float(w * h)
    return {"psnr_db": p, "bytes": len(blob), "bpp": bpp, "rd_score": rate.rd_score(p, len(blob), w, h, quality)}
