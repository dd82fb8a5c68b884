"""HDF5 files without libhdf5: the library's writer (cb_h5_write_floats).

The reference stores field snapshots through the HDF5 C++ library
(Bubble::OutField, src/bubble.cpp:919-953). This build writes the same kind
of file itself; see coolbubble_b200/csrc/cb_h5.cpp for the format.
"""
from __future__ import annotations

import os

import numpy as np

from . import _lib as L


def write_floats(path, datasets, chunks, attrs=None, deflate_level=9, threads=0):
    """Write float32 datasets of one shape, chunked with `chunks`, shuffled and
    deflated, plus scalar double attributes on the root group.

    datasets: {name: array} (all the same shape, rank 1-3, cast to float32);
    attrs: {name: float}. Raises CBError on a bad argument or a write error.
    """
    names = list(datasets)
    arrays = [np.ascontiguousarray(datasets[k], dtype=np.float32) for k in names]
    if not arrays:
        raise ValueError("no datasets")
    shape = arrays[0].shape
    if any(a.shape != shape for a in arrays):
        raise ValueError("datasets differ in shape")
    rank = len(shape)
    chunks = tuple(int(c) for c in chunks)
    if len(chunks) != rank:
        raise ValueError("chunks must have one entry per dimension")
    attrs = dict(attrs or {})
    dims = (L.C.c_int64 * rank)(*shape)
    ch = (L.C.c_int64 * rank)(*chunks)
    nm = (L.C.c_char_p * len(names))(*[k.encode() for k in names])
    dp = (L._fp * len(arrays))(*[L.fptr(a) for a in arrays])
    an = (L.C.c_char_p * max(1, len(attrs)))(*[k.encode() for k in attrs])
    av = np.array([float(v) for v in attrs.values()] or [0.0])
    L.check(L.lib.cb_h5_write_floats(os.fsencode(path), rank, dims, ch, len(names), nm, dp, len(attrs), an,
                                     L.dptr(av), int(deflate_level), int(threads)))
