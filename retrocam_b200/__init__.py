"""retrocam_b200 -- B200-native render hot path of RetroCam.

The product is libretrocam.so (built from retrocam_b200/csrc by
retrocam_b200.build) behind the C ABI in include/retrocam.h; `api` is its
Python binding and a mirror of the reference's Java render-path classes;
`scenes` describes the benchmark workloads.
"""
from . import scenes  # noqa: F401

__all__ = ["scenes", "api", "build"]
