"""weft_b200 — B200 (sm_100a) kernels for Weft's primitive-stack hot path.

Modules:
  gpu_render  drop-in replacements of the reference's GPU render/score launchers
  fit         batched, device-resident greedy candidate-scoring fit
  refine      hand-written backward + Adam refinement of fitted stacks
  render      the decoder's primitive walk on the GPU
  raster      the decoder's raster branch: DCT residual layer and u8 BILINEAR resize on the GPU
  candidates  the reference's candidate generators (host, numpy)
  quadtree    tile layout; rate: lambda / bits / RD score; synth: test images
"""

__all__ = ["install_into", "install_raster_into"]


def install_into(gpu_render_module) -> None:
    """Replace the reference's launchers in ``gpu_render_module`` (``weft.gpu_render``).

    The reference imports its launchers inside the calling functions
    (src/weft/encoder.py:2655), so the swap takes effect on the next call.
    """
    from . import gpu_render as g

    for name in ("gpu_batch_score_prepacked", "gpu_batch_objectives", "gpu_render_tiles_to_image"):
        setattr(gpu_render_module, name, getattr(g, name))


def install_raster_into(dct_residual_module) -> None:
    """Replace ``apply_residual_to_image`` in ``dct_residual_module`` (``weft.dct_residual``) with the
    GPU layer.  The reference decoder imports it inside its DCT branch (src/weft/decoder.py:477-486),
    so the swap takes effect on the next decode."""
    from . import raster

    dct_residual_module.apply_residual_to_image = raster.apply_residual_to_image
