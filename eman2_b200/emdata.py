"""EMData: a minimal image container for the reconstruction API.

Holds a float32 numpy array and an attribute dict, with the accessors the
reconstruction path uses (EMData::get_attr/set_attr/has_attr,
libEM/emdata_metadata.cpp:1006-1143; sizes; complex flag).  A complex image
stores the reference's r2c layout: float[ny][nx] with nx = N+2 interleaved
re/im pairs.
"""
from __future__ import annotations

import numpy as np

from .exceptions import NotExistingObjectException


class EMData:
    def __init__(self, data=None, nx=None, ny=None, nz=1, is_complex=False, attrs=None):
        if data is None:
            shape = (ny or 1, nx or 1) if nz == 1 else (nz, ny or 1, nx or 1)
            data = np.zeros(shape, np.float32)
        if hasattr(data, "detach"):
            data = data.detach().cpu().numpy()
        self._data = np.ascontiguousarray(data, np.float32)
        self._complex = bool(is_complex)
        self.attrs = {"apix_x": 1.0, "apix_y": 1.0, "apix_z": 1.0}
        if attrs:
            self.attrs.update(attrs)

    # ------------------------------------------------------------- data
    def numpy(self) -> np.ndarray:
        return self._data

    def get_data(self) -> np.ndarray:
        return self._data

    def set_data(self, a):
        self._data = np.ascontiguousarray(a, np.float32)

    def is_complex(self) -> bool:
        return self._complex

    def get_xsize(self) -> int:
        return int(self._data.shape[-1])

    def get_ysize(self) -> int:
        return int(self._data.shape[-2]) if self._data.ndim >= 2 else 1

    def get_zsize(self) -> int:
        return int(self._data.shape[-3]) if self._data.ndim >= 3 else 1

    def copy(self) -> "EMData":
        return EMData(self._data.copy(), is_complex=self._complex, attrs=dict(self.attrs))

    def complex_view(self) -> np.ndarray:
        """The complex64 view of a complex image (..., nx/2)."""
        return self._data.view(np.complex64)

    # ------------------------------------------------------------- attributes
    def get_attr(self, key):
        if key not in self.attrs:
            raise NotExistingObjectException(f"The requested key does not exist: {key}")
        return self.attrs[key]

    def get_attr_default(self, key, default=None):
        return self.attrs.get(key, default)

    def set_attr(self, key, value):
        self.attrs[key] = value

    def has_attr(self, key) -> bool:
        return key in self.attrs

    def __getitem__(self, key):
        if key == "nx":
            return self.get_xsize()
        if key == "ny":
            return self.get_ysize()
        if key == "nz":
            return self.get_zsize()
        return self.get_attr(key)

    def __setitem__(self, key, value):
        self.set_attr(key, value)

    def __repr__(self):
        kind = "complex" if self._complex else "real"
        return f"EMData({kind} {self.get_xsize()}x{self.get_ysize()}x{self.get_zsize()})"
