"""eman2_b200 -- EMAN2's direct Fourier inversion (FourierReconstructor,
Reconstructors.get("fourier")) on B200 GPUs.

Public API mirrors the reference:

    from eman2_b200 import Reconstructors, Transform, EMData
    recon = Reconstructors.get("fourier", {"size": [N]*3, "sym": "d7", "mode": "gauss_5"})
    recon.setup()
    recon.insert_slice(img, xform, weight)
    recon.determine_slice_agreement(img, xform, weight, False)
    vol = recon.finish(True)

plus batched forms (``insert_slices``, ``insert_particles``), many
reconstructions per launch (``eman2_b200.batch``) and a serving loop
(``eman2_b200.server``).  The compute runs in libeman2_b200.so (CUDA for
sm_100a) through a C ABI (include/eman2_b200.h).
"""
from .emdata import EMData, Region
from .exceptions import (DeviceException, ImageDimensionException, InvalidParameterException,
                         NotExistingObjectException, NullPointerException, StateException,
                         UnsupportedParameterException)
from .reconstructor import (FourierIterReconstructor, FourierReconstructor, Reconstructors,
                            WienerFourierReconstructor)
from .transform import Transform

__all__ = [
    "EMData", "Region", "Transform", "Reconstructors", "FourierReconstructor",
    "WienerFourierReconstructor", "FourierIterReconstructor",
    "InvalidParameterException", "ImageDimensionException", "NullPointerException",
    "NotExistingObjectException", "StateException", "DeviceException",
    "UnsupportedParameterException",
]
