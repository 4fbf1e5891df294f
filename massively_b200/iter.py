"""zip2..zip12: row views over several columns (massively/src/api/iter.rs:1169-1330)."""
from __future__ import annotations

import numpy as np


class Zip:
    """Columns read (and written) together as rows; all of one length."""

    def __init__(self, *cols):
        if not 1 <= len(cols) <= 12:
            raise ValueError("a zip holds 1 to 12 columns")
        n = len(cols[0])
        for c in cols[1:]:
            if len(c) != n:
                from .runtime import LengthMismatch
                raise LengthMismatch(n, len(c))
        self.cols = list(cols)

    def __len__(self):
        return len(self.cols[0])

    def __iter__(self):
        return iter(self.cols)

    def __getitem__(self, k):
        return self.cols[k]

    @property
    def dtype(self):
        return np.dtype([(f"c{k}", c.dtype) for k, c in enumerate(self.cols)])

    def into_columns(self):
        """MStorage::into_columns."""
        return tuple(self.cols)


def _zipn(n):
    def z(*cols):
        if len(cols) != n:
            raise TypeError(f"zip{n} takes {n} columns")
        return Zip(*cols)
    z.__name__ = f"zip{n}"
    z.__doc__ = f"zip{n}: a {n}-column row view."
    return z


zip2, zip3, zip4, zip5, zip6, zip7, zip8, zip9, zip10, zip11, zip12 = (_zipn(k) for k in range(2, 13))
