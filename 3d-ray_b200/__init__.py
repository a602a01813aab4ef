"""B200-native path-tracing core for 3d-ray (loaded under the module name
`rt3d_b200`; the directory name is not a Python identifier)."""
from . import abi, adjoint, images, objfile, renderer, scenes  # noqa: F401
from .adjoint import DiffScene  # noqa: F401
from .renderer import RenderBuffers, RenderCaptureOptions, Renderer, RenderResult, render_batch  # noqa: F401
