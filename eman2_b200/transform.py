"""Transform: the subset of EMAN2's Transform used by the reconstruction path.

A 3x4 float32 matrix [R | t] built the way libEM/transform.cpp builds it:
Euler conversions in double precision with libm trigonometry, each element
rounded to float once (Transform::set_rotation, libEM/transform.cpp:527-700);
the product of two transforms in float (EMAN::operator*, :1384-1395); the
inverse through double cofactors (Transform::invert, :1324-1356).
"""
from __future__ import annotations

import math

import numpy as np

_DEG2RAD = 3.141592653589793238462643383279502884197169399 / 180.0
_ROT_KEYS = {
    "2d": ("alpha",), "eman": ("az", "alt", "phi"), "imagic": ("alpha", "beta", "gamma"),
    "spider": ("phi", "theta", "psi"), "mrc": ("phi", "theta", "omega"),
    "xyz": ("xtilt", "ytilt", "ztilt"), "quaternion": ("e0", "e1", "e2", "e3"),
    "spin": ("omega", "n1", "n2", "n3"), "spinvec": ("v1", "v2", "v3"),
    "sgirot": ("q", "n1", "n2", "n3"),
    "matrix": ("m11", "m12", "m13", "m21", "m22", "m23", "m31", "m32", "m33"),
}
_f32 = np.float32


def _eman(az, alt, phi):
    azp, altp, phip = az * _DEG2RAD, alt * _DEG2RAD, phi * _DEG2RAD
    c, s = math.cos, math.sin
    return [
        [c(phip) * c(azp) - c(altp) * s(azp) * s(phip),
         c(phip) * s(azp) + c(altp) * c(azp) * s(phip),
         s(altp) * s(phip)],
        [-s(phip) * c(azp) - c(altp) * s(azp) * c(phip),
         -s(phip) * s(azp) + c(altp) * c(azp) * c(phip),
         s(altp) * c(phip)],
        [s(altp) * s(azp), -s(altp) * c(azp), c(altp)],
    ]


def _quat(e0, e1, e2, e3):
    return [
        [e0 * e0 + e1 * e1 - e2 * e2 - e3 * e3, 2.0 * (e1 * e2 + e0 * e3), 2.0 * (e1 * e3 - e0 * e2)],
        [2.0 * (e2 * e1 - e0 * e3), e0 * e0 - e1 * e1 + e2 * e2 - e3 * e3, 2.0 * (e2 * e3 + e0 * e1)],
        [2.0 * (e3 * e1 + e0 * e2), 2.0 * (e3 * e2 - e0 * e1), e0 * e0 - e1 * e1 - e2 * e2 + e3 * e3],
    ]


class Transform:
    """3x4 transform [R | t] (row-major, float32)."""

    def __init__(self, arg=None):
        self.matrix = np.zeros((3, 4), np.float32)
        self.matrix[0, 0] = self.matrix[1, 1] = self.matrix[2, 2] = 1.0
        if arg is None:
            return
        if isinstance(arg, Transform):
            self.matrix = arg.matrix.copy()
        elif isinstance(arg, dict):
            self.set_params(arg)
        else:
            a = np.asarray(arg, np.float32).reshape(-1)
            if a.size == 12:
                self.matrix = a.reshape(3, 4).copy()
            elif a.size == 9:
                self.matrix[:, :3] = a.reshape(3, 3)
            else:
                raise ValueError("Transform takes a dict, 9 or 12 numbers")

    # ---------------------------------------------------------------- params
    def set_params(self, d: dict):
        d = {k.lower(): v for k, v in d.items()}
        if "type" in d:
            self.set_rotation(d)
        if "scale" in d and float(d["scale"]) != 1.0:
            raise ValueError("scaled transforms are outside the reconstruction path")
        tx, ty, tz = (float(d.get(k, 0.0)) for k in ("tx", "ty", "tz"))
        if tx or ty or tz:
            self.set_trans(tx, ty, tz)
        if d.get("mirror"):
            raise ValueError("mirrored transforms are outside the reconstruction path")

    def set_rotation(self, d: dict):
        d = {k.lower(): v for k, v in d.items()}
        kind = str(d.get("type", "")).lower()
        if kind not in _ROT_KEYS:
            raise ValueError(f"unknown Euler type {kind!r}")
        g = lambda k: float(d.get(k, 0.0))  # noqa: E731
        if kind == "eman":
            m = _eman(g("az"), g("alt"), g("phi"))
        elif kind == "2d":
            m = _eman(0.0, 0.0, g("alpha"))
        elif kind == "imagic":
            m = _eman(g("alpha"), g("beta"), g("gamma"))
        elif kind == "spider":
            m = _eman(g("phi") + 90.0, g("theta"), g("psi") - 90.0)
        elif kind == "mrc":
            m = _eman(g("phi") + 90.0, g("theta"), g("omega") - 90.0)
        elif kind == "quaternion":
            m = _quat(g("e0"), g("e1"), g("e2"), g("e3"))
        elif kind == "spin":
            n1, n2, n3 = g("n1"), g("n2"), g("n3")
            norm = math.sqrt(n1 * n1 + n2 * n2 + n3 * n3)
            if norm == 0.0:
                m = _quat(1.0, 0.0, 0.0, 0.0)
            else:
                om = g("omega") * _DEG2RAD / 2.0
                m = _quat(math.cos(om), math.sin(om) * n1 / norm, math.sin(om) * n2 / norm,
                          math.sin(om) * n3 / norm)
        elif kind == "spinvec":
            v1, v2, v3 = g("v1"), g("v2"), g("v3")
            ln = math.sqrt(v1 * v1 + v2 * v2 + v3 * v3)
            if ln == 0.0:
                m = _quat(1.0, 0.0, 0.0, 0.0)
            else:
                om = 2.0 * math.pi * ln
                m = _quat(math.cos(om / 2), math.sin(om / 2) * v1 / ln,
                          math.sin(om / 2) * v2 / ln, math.sin(om / 2) * v3 / ln)
        elif kind == "sgirot":
            om = g("q") * _DEG2RAD / 2.0
            m = _quat(math.cos(om), math.sin(om) * g("n1"), math.sin(om) * g("n2"),
                      math.sin(om) * g("n3"))
        elif kind == "xyz":
            cx, sx = math.cos(_DEG2RAD * g("xtilt")), math.sin(_DEG2RAD * g("xtilt"))
            cy, sy = math.cos(_DEG2RAD * g("ytilt")), math.sin(_DEG2RAD * g("ytilt"))
            cz, sz = math.cos(_DEG2RAD * g("ztilt")), math.sin(_DEG2RAD * g("ztilt"))
            m = [[cy * cz, cx * sz + sx * sy * cz, sx * sz - cx * sy * cz],
                 [-cy * sz, cx * cz - sx * sy * sz, sx * cz + cx * sy * sz],
                 [sy, -sx * cy, cx * cy]]
        else:  # matrix
            m = [[g("m11"), g("m12"), g("m13")], [g("m21"), g("m22"), g("m23")],
                 [g("m31"), g("m32"), g("m33")]]
        self.matrix[:, :3] = np.array(m, np.float64).astype(np.float32)

    def set_trans(self, x, y=0.0, z=0.0):
        self.matrix[:, 3] = np.array([x, y, z], np.float32)

    def get_trans(self):
        return [float(v) for v in self.matrix[:, 3]]

    def get_trans_2d(self):
        return [float(self.matrix[0, 3]), float(self.matrix[1, 3])]

    def get_matrix(self):
        return [float(v) for v in self.matrix.reshape(-1)]

    def rotation_block(self) -> np.ndarray:
        return np.ascontiguousarray(self.matrix[:, :3])

    def get_rotation(self, kind: str = "eman") -> dict:
        """Euler angles ("eman") of the rotation (libEM/transform.cpp:852-905)."""
        if kind.lower() != "eman":
            raise ValueError("only the eman convention is provided")
        m = self.matrix.astype(np.float64)
        cosalt = m[2, 2]
        if cosalt >= 1:
            return {"type": "eman", "az": 0.0, "alt": 0.0,
                    "phi": math.degrees(math.atan2(m[0, 1], m[0, 0]))}
        if cosalt <= -1:
            return {"type": "eman", "az": 0.0, "alt": 180.0,
                    "phi": math.degrees(math.atan2(-m[0, 1], m[0, 0]))}
        az = math.degrees(math.atan2(m[2, 0], -m[2, 1]))
        alt = 90.0 if m[2, 2] == 0 else math.degrees(
            math.atan(math.sqrt(m[2, 0] ** 2 + m[2, 1] ** 2) / abs(m[2, 2])))
        if m[2, 2] < 0:
            alt = 180.0 - alt
        phi = math.degrees(math.atan2(m[0, 2], m[1, 2]))
        return {"type": "eman", "az": az, "alt": alt, "phi": phi}

    # ---------------------------------------------------------------- algebra
    def invert(self):
        m = self.matrix.astype(np.float64)
        m00, m01, m02, v0 = m[0]
        m10, m11, m12, v1 = m[1]
        m20, m21, m22, v2 = m[2]
        cof00 = m11 * m22 - m12 * m21
        cof11 = m22 * m00 - m20 * m02
        cof22 = m00 * m11 - m01 * m10
        cof01 = m10 * m22 - m20 * m12
        cof02 = m10 * m21 - m20 * m11
        cof12 = m00 * m21 - m01 * m20
        cof10 = m01 * m22 - m02 * m21
        cof20 = m01 * m12 - m02 * m11
        cof21 = m00 * m12 - m10 * m02
        det = m00 * cof00 + m02 * cof02 - m01 * cof01
        out = np.array([
            [cof00 / det, -(np.float32(cof10 / det)), cof20 / det,
             (-cof00 * v0 + cof10 * v1 - cof20 * v2) / det],
            [-(np.float32(cof01 / det)), cof11 / det, -(np.float32(cof21 / det)),
             (cof01 * v0 - cof11 * v1 + cof21 * v2) / det],
            [cof02 / det, -(np.float32(cof12 / det)), cof22 / det,
             (-cof02 * v0 + cof12 * v1 - cof22 * v2) / det],
        ], np.float64)
        self.matrix = out.astype(np.float32)
        return self

    def inverse(self) -> "Transform":
        return Transform(self).invert()

    def __mul__(self, other: "Transform") -> "Transform":
        a, b = self.matrix, other.matrix
        r = Transform()
        for i in range(3):
            for j in range(4):
                v = _f32(a[i, 0]) * _f32(b[0, j])
                v = _f32(v + _f32(a[i, 1]) * _f32(b[1, j]))
                v = _f32(v + _f32(a[i, 2]) * _f32(b[2, j]))
                r.matrix[i, j] = v
            r.matrix[i, 3] = _f32(r.matrix[i, 3] + a[i, 3])
        return r

    def is_identity(self) -> bool:
        m = self.matrix
        for i in range(3):
            for j in range(4):
                c = float(m[i, j])
                if abs(c - math.ceil(c)) < 1e-6:
                    c = math.ceil(c)
                elif abs(c - math.floor(c)) < 1e-6:
                    c = math.floor(c)
                if c != (1.0 if i == j else 0.0):
                    return False
        return True

    def __repr__(self):
        return f"Transform({self.get_matrix()})"


def quaternion_to_transform(q) -> Transform:
    return Transform({"type": "quaternion", "e0": float(q[0]), "e1": float(q[1]),
                      "e2": float(q[2]), "e3": float(q[3])})
