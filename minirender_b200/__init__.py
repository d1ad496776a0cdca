"""B200-native offline path tracer with MiniRender's scene, camera and render-settings interface.

``minirender_b200.scene`` builds scene documents and snapshots (pure Python/numpy).
``minirender_b200.api`` is the host mirror of the reference's ``PathTracer`` and
``RenderSession`` over the C ABI of ``libminirender_b200.so`` (CUDA, sm_100a).
"""

from . import scene  # noqa: F401

__all__ = ["scene", "api"]
