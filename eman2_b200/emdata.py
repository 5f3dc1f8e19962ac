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


class Region:
    """Region(x0, y0, z0, nx, ny, nz) (libEM/geometry.h)."""

    def __init__(self, x0, y0, z0=0, nx=1, ny=1, nz=1):
        self.origin = (int(x0), int(y0), int(z0))
        self.size = (int(nx), int(ny), int(nz))


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

    # ------------------------------------------------------------- processing
    def process_inplace(self, name: str, params: dict | None = None):
        """EMData::process_inplace for the processors this path uses:
        math.gausskernelfix (MaskGaussInvProcessor, libEM/processor.h:4131-4176),
        run on the GPU."""
        params = params or {}
        if name == "math.gausskernelfix":
            if self._complex:
                return        # CoordinateProcessor::is_valid: real images only
            from . import _lib
            _lib.check(_lib.load().fr_kernel_fix(
                _lib.ptr(self._data), self.get_xsize(), self.get_ysize(), self.get_zsize(),
                float(params.get("gauss_width", 0.0)), None))
            return
        raise NotExistingObjectException(f"No such an instance existing: {name}")

    def clip_inplace(self, region: "Region"):
        """EMData::clip_inplace to a region inside the image (zero fill outside)."""
        x0, y0, z0, nx, ny, nz = region.origin + region.size
        src = self._data if self._data.ndim == 3 else self._data[None]
        out = np.zeros((nz, ny, nx), np.float32)
        zs, ys, xs = src.shape
        sz = slice(max(0, z0), min(zs, z0 + nz)); sy = slice(max(0, y0), min(ys, y0 + ny))
        sx = slice(max(0, x0), min(xs, x0 + nx))
        out[sz.start - z0:sz.stop - z0, sy.start - y0:sy.stop - y0, sx.start - x0:sx.stop - x0] = \
            src[sz, sy, sx]
        self._data = out if self._data.ndim == 3 else out[0]

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
