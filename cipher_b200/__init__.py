"""cipher_b200 - B200 implementation of CIPHER's time-stepper right-hand side.

The compute path is the CUDA library ``libcipher_b200.so`` (sm_100a) behind
the C ABI of ``include/cipher_b200.h``; this package is its Python face.
"""
from ._lib import CipherError, load  # noqa: F401
from .api import (AMR, Batch, Config, Context, Forest, Mesh, Nucleation, Problem, Server, TimeStepper, TSView, diffuse_state_aos,  # noqa: F401
                  compute_output, initial_state_aos, nuclei_array, ts_options, write_vtu)

__all__ = ["AMR", "Batch", "CipherError", "Config", "Forest", "Nucleation", "Context", "Mesh", "Problem", "Server", "TimeStepper", "TSView", "diffuse_state_aos",
           "compute_output", "initial_state_aos", "nuclei_array", "load", "ts_options", "write_vtu"]
