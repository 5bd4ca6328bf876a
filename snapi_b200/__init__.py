"""snapi_b200 -- B200 (sm_100a) implementation of SNAPI's per-pixel Stokes synthesis, node
responses, chi2 adjoint gradient, LM node fit and NLTE level populations, behind the C ABI libsnapi_cuda
(include/snapi_cuda.h).  This package holds the CUDA sources (csrc/), the build step and a
Python mirror of the C ABI for tests and benchmarks."""
from .api import (Context, SnapiError, SnapiLine, lib, lines_from_arrays, zeeman_pattern,  # noqa: F401
                  MEM_DEVICE, MEM_HOST, NFIELD0, FIELD_NAMES, AliContext, pack_tangents, tangent_field_mask,
                  f0_read, f0_stat, f0_write)

__all__ = ["Context", "SnapiError", "SnapiLine", "lib", "lines_from_arrays", "zeeman_pattern", "MEM_DEVICE",
           "MEM_HOST", "NFIELD0", "FIELD_NAMES", "AliContext", "pack_tangents", "tangent_field_mask", "f0_read",
           "f0_stat", "f0_write"]
