"""B200-native pseudo-spectral Galerkin Couette step (jaxfun drop-in).

Hand-written sm_100a CUDA behind the C ABI in ``include/jfb200.h``; this
package is the Python host side mirroring the reference's API.
"""

__version__ = "0.1.0"
