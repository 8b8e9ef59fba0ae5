"""idx2_b200: the idx2 encode/decode hot path on NVIDIA B200 (sm_100a).

Python mirror of the reference's encode/decode interface over the C ABI in
``include/idx2g.h`` (libidx2g.so, built in-tree by ``__graft_entry__.build()``).
The compute path is the CUDA library; there is no CPU fallback: if the library
or a GPU is missing, every call raises.

    >>> import idx2_b200 as idx2
    >>> idx2.encode(field, out_dir="out", name="Miranda", field_name="Density",
    ...             num_levels=2, tolerance=1e-3)
    >>> ds = idx2.Dataset("out/Miranda/Density.idx2")
    >>> grid = ds.decode(downsampling=(1, 1, 1), tolerance=1e-3)
"""
from __future__ import annotations

from ._lib import (Idx2Error, Params, check_params, encode, encode_batch, encode_device, lib, lib_path,
                   ctx, error_string)
from .dataset import Dataset

__all__ = ["Idx2Error", "Params", "check_params", "encode", "encode_batch", "encode_device", "lib", "lib_path", "ctx",
           "error_string", "Dataset"]
