"""magnet_b200 — MAGNET's layout pass on one B200 (sm_100a).

The device path is the compiled library ``libmagnet_b200.so`` (C ABI, include/magnet_b200.h) and its pybind11
surface ``magnet_b200._native``, which carries the names and arguments of the reference's native module
``_magnet`` (kerighan/lib-magnet, src/bindings.cpp). There is no CPU fallback: importing this package raises if
the native library is missing or was built for another architecture.

Python-level drivers, mirroring the reference's:
  * ``optimize_tsne``      magnet/tsne.py:132-214 (the whole loop on the device, CUDA-graph replayed)
  * ``optimize_tsne_batch`` many such loops together, one graph per iteration (magnet_b200.autotune sizes it)
  * ``FFTRepulsion2D``     magnet/tsne.py:11-129 (grid choice, cached kernel spectra, FFTConv2D objects)
  * ``optimize_sgd``       MAGNET._optimize, magnet/__init__.py:751-869 (segments, linear schedules)
  * ``edge_schedule``      magnet/__init__.py:51-66, 727-737
  * ``hybrid_layout``      the loss="hybrid" sequence, magnet/__init__.py:683-708
  * ``transform_layout``   the out-of-sample SGD of MAGNET.transform, magnet/__init__.py:896-930
"""
import os

from . import _native  # noqa: F401  (raises ImportError loudly when the extension is missing)
from ._native import (FFTConv2D, optimize_layout, tsne_attraction, tsne_step, tsne_update, bbox_2d,  # noqa: F401
                      mid_spring, layout_schedule, synchronize, set_stream, center_scale, launch_count,
                      optimize_tsne_profiled)
from .drivers import (FFTRepulsion2D, optimize_tsne, optimize_tsne_batch, optimize_sgd, edge_schedule,  # noqa: F401
                      sampling_frequencies, hybrid_layout, transform_layout, find_ab_params)

__version__ = "0.1.0"
LIBRARY = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "libmagnet_b200.so")
