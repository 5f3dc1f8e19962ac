"""Exception classes named after the reference's (libEM/exception.h), raised
for the C ABI's status codes."""
from __future__ import annotations


class EMANException(RuntimeError):
    """Base of the library's errors."""


class InvalidParameterException(EMANException):
    """Unknown or malformed parameter (libEM/emobject.h:931-938)."""


class ImageDimensionException(EMANException):
    """Image or volume sizes do not fit (libEM/reconstructor.cpp:767,861)."""


class NullPointerException(EMANException):
    """A required image is missing (libEM/reconstructor.cpp:1067)."""


class NotExistingObjectException(EMANException):
    """A required attribute is missing (libEM/emdata_metadata.cpp:1142)."""


class InvalidValueException(EMANException):
    """A value outside its allowed range."""


class UnsupportedParameterException(EMANException):
    """A parameter value the reference accepts but this build does not cover."""


class StateException(EMANException):
    """The reconstructor was used before setup() or after finish()."""


class DeviceException(EMANException):
    """CUDA runtime, cuFFT or kernel failure."""


_BY_STATUS = {
    1: InvalidParameterException,
    2: ImageDimensionException,
    3: NullPointerException,
    4: StateException,
    5: DeviceException,
    6: DeviceException,
    7: UnsupportedParameterException,
    8: NotExistingObjectException,
    9: DeviceException,
}


def raise_status(code: int, message: str):
    raise _BY_STATUS.get(code, EMANException)(message or f"status {code}")
