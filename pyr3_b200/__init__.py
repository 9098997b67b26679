"""pyr3-b200: a B200-native fractal-flame engine (chaos game -> u32
histogram -> density estimation -> tonemap) behind the reference pyr3
Renderer API, with hand-written CUDA for sm_100a behind a C-ABI
(include/pyr3.h, libpyr3cuda.so)."""
from .genome import Genome, Variation, Xform, bake_lut, genome_from_json, genome_to_json  # noqa: F401
from .renderer import Renderer, compute_dispatch, create_renderer  # noqa: F401
