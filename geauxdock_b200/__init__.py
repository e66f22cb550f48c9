"""geauxdock_b200 -- B200 (sm_100a) Monte Carlo docking backend with the
GeauxDock Dock(...) boundary.

The product is libgdock.so (CUDA kernels + C ABI, include/gdock.h); this
package holds its sources (csrc/), the build script, and the Python host
mirror used by tests and benchmarks: ctypes bindings (_lib), numpy mirrors of
the boundary structs (layout), the force-field parameters (params), the
synthetic complex generator (synth) and the reference-style Dock driver
(dock).
"""

from ._lib import GdockError, load  # noqa: F401

__all__ = ["GdockError", "load"]
