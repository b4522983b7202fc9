"""weft_b200 — B200 (sm_100a) kernels for Weft's primitive-stack hot path.

Modules:
  gpu_render  drop-in replacements of the reference's GPU render/score launchers
  fit         batched, device-resident greedy candidate-scoring fit
  refine      hand-written backward + Adam refinement of fitted stacks
  render      the decoder's primitive walk on the GPU
  candidates  the reference's candidate generators (host, numpy)
  quadtree    tile layout; rate: lambda / bits / RD score; synth: test images
"""

__all__ = ["install_into"]


def install_into(gpu_render_module) -> None:
    """Replace the reference's launchers in ``gpu_render_module`` (``weft.gpu_render``).

    The reference imports its launchers inside the calling functions
    (src/weft/encoder.py:2655), so the swap takes effect on the next call.
    """
    from . import gpu_render as g

    for name in ("gpu_batch_score_prepacked", "gpu_batch_objectives", "gpu_render_tiles_to_image"):
        setattr(gpu_render_module, name, getattr(g, name))
