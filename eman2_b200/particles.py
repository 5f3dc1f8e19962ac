"""Per-particle metadata for the batched caller pipeline (fr_particle)."""
from __future__ import annotations

import numpy as np

from . import _lib


def particle_meta(rots, shifts=None, weights=None, ctf: dict | None = None, defocus=None,
                  apix: float = 1.0):
    """Build a ctypes array of ``fr_particle``.

    rots: (n, 3, 3) rotation blocks of xform.projection; shifts: (n, 2)
    translations of xform.projection; weights: (n,); ctf: common CTF fields
    (voltage kV, cs mm, ampcont %, apix, dfdiff, dfang); defocus: (n,) in um
    (|defocus| <= 1e-4 or None: no phase flip)."""
    rots = np.asarray(rots, np.float32).reshape(-1, 9)
    n = rots.shape[0]
    shifts = np.zeros((n, 2), np.float32) if shifts is None else np.asarray(shifts, np.float32)
    weights = np.ones(n, np.float32) if weights is None else np.asarray(weights, np.float32)
    defocus = np.zeros(n, np.float32) if defocus is None else np.asarray(defocus, np.float32)
    c = {"voltage": 300.0, "cs": 2.7, "ampcont": 10.0, "apix": apix, "dfdiff": 0.0, "dfang": 0.0}
    if ctf:
        c.update(ctf)
    arr = (_lib.fr_particle * n)()
    for i in range(n):
        p = arr[i]
        for k in range(9):
            p.rot[k] = float(rots[i, k])
        p.tx, p.ty = float(shifts[i, 0]), float(shifts[i, 1])
        p.weight = float(weights[i])
        p.defocus = float(defocus[i])
        p.dfdiff, p.dfang = float(c["dfdiff"]), float(c["dfang"])
        p.voltage, p.cs = float(c["voltage"]), float(c["cs"])
        p.apix, p.ampcont = float(c["apix"]), float(c["ampcont"])
    return arr
