"""The two-electron part of the TREXIO export, host side.

trexio_conv_integrals (src/trexio/trexio_conv.f90:267-359) writes the
integrals to a TREXIO file in buffers: it walks (i, j, k, l), i fastest,
keeps the entries with i >= j, (i == j => k >= l) and ERI(i, k, j, l) != 0,
and every BUFSIZE = 10000 entries calls trexio_write_ao_2e_int_eri(file,
offset, BUFSIZE, index, values).  The device produces that entry stream
(tce_trexio_eri, `Engine.trexio_eri`); `eri_chunks` cuts it into the
reference's calls.  libtrexio (and its HDF5 back end) is not available here,
so no TREXIO file is written: the calls are returned for a caller that links
libtrexio.

Two details of the reference are kept as they are: the last, partial buffer
is passed with count BUFSIZE rather than the number of new entries (:353), so
its tail repeats entries of the previous buffer (the reference's buffers are
never cleared; before the first full buffer they hold whatever the stack
held, zeros here); and the routine needs the full nbas^4 array, so a run in
SAO mode has no two-electron export.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

BUFSIZE = 10000


def eri_chunks(index: np.ndarray, value: np.ndarray, bufsize: int = BUFSIZE
               ) -> List[Tuple[int, int, np.ndarray, np.ndarray]]:
    """The trexio_write_ao_2e_int_eri calls of the reference for an entry
    stream: (offset, count, index[count, 4], value[count]) per call."""
    index = np.asarray(index, dtype=np.int32).reshape(-1, 4)
    value = np.asarray(value, dtype=np.float64)
    n = len(value)
    buf_i = np.zeros((bufsize, 4), dtype=np.int32)
    buf_v = np.zeros(bufsize)
    calls = []
    offset = 0
    for c0 in range(0, n, bufsize):
        m = min(bufsize, n - c0)
        buf_i[:m] = index[c0:c0 + m]
        buf_v[:m] = value[c0:c0 + m]
        calls.append((offset, bufsize, buf_i.copy(), buf_v.copy()))
        if m == bufsize:
            offset += m
    return calls


def reference_stream(eri: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """The entry stream written out directly from a full ERI(n, n, n, n) array
    (column-major, as the reference holds it), for checks."""
    n = eri.shape[0]
    i, j, k, l = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    # loop order: i fastest, then j, k, l  ->  flatten in Fortran order of (i, j, k, l)
    i, j, k, l = (x.ravel(order="F") for x in (i, j, k, l))
    v = eri[i, k, j, l]
    keep = (i >= j) & ~((i == j) & (k < l)) & (v != 0.0)
    idx = np.stack([i[keep] + 1, j[keep] + 1, k[keep] + 1, l[keep] + 1], axis=1).astype(np.int32)
    return idx, v[keep]
