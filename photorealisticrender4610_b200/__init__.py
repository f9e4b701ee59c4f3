"""B200-native (sm_100a) Monte Carlo path-tracing hot path of the
PhotoRealisticRender4610 renderer: SAH-BVH traversal, the path integrator,
environment-map importance sampling, caustic photons and tone mapping as
hand-written CUDA behind a C ABI (include/prr.h), with a Python mirror of the
reference's Scene / BVHAccel / Integrator / Renderer interface."""
from ._lib import PrrError, header_symbols, load  # noqa: F401
from . import scenes  # noqa: F401
from .api import (PhotonMap, Scene, Server, medium_intersect, medium_preset,  # noqa: F401
                  phase_hg, phase_hg_sample, read_obj, sample_count_image, tonemap,
                  write_image)

__all__ = ["Scene", "PhotonMap", "Server", "PrrError", "load", "header_symbols", "scenes",
           "tonemap"]
