"""B200-native adjoint renderer for beta surfels.

``differentiablepointrendering_b200.pale`` is the drop-in ``pale`` module
(``pale.Renderer``); ``scene`` builds scene descriptions; ``autograd``
wraps the renderer as a ``torch.autograd.Function``.
"""
from .scene import SceneArrays, make_box_scene, make_surfels, jitter_target  # noqa: F401

__all__ = ["SceneArrays", "make_box_scene", "make_surfels", "jitter_target"]
