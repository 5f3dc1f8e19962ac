"""Reconstructors.get("fourier", {...}) -- the drop-in for EMAN2's
FourierReconstructor (libEM/reconstructor.h:388-565, libEM/reconstructor.cpp:686-1641)
and its Python binding (libpyEM/libpyReconstructor2.cpp:192-226).

Same method names, parameter keys, defaults, return values and exception
classes; the work runs on the GPU through libeman2_b200.so.  Images may be
``EMData`` objects, numpy arrays or torch tensors (host or CUDA; CUDA tensors
are used in place).
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _lib
from .emdata import EMData
from .exceptions import (ImageDimensionException, InvalidParameterException,
                         NotExistingObjectException, NullPointerException, StateException,
                         UnsupportedParameterException)
from .transform import Transform

# FourierReconstructor::get_param_types (libEM/reconstructor.h:501-516).
PARAM_TYPES = {
    "size": ("INTARRAY", "Required. The dimensions of the real-space output volume, including any "
             "padding (must be handled by the calling application). Assumed that apix x/y/z "
             "identical."),
    "sym": ("STRING", "Required. The symmetry of the reconstructed volume, c?, d?, oct, tet, icos, "
            "h?. Default is c1, ie - an asymmetric object"),
    "mode": ("STRING", "Optional. Fourier pixel insertion mode name (nearest_neighbor, gauss_2, "
             "gauss_3, gauss_5, gauss_5_slow, gypergeom_5, experimental) gauss_2 is the default."),
    "corners": ("BOOL", "Optional. If not set, then reconstruction will cover a spherical volume "
                "with a radius of nx/2. If set, the full Fourier volume will be reconstructed, but "
                "will be ~2x slower."),
    "sqrtnorm": ("BOOL", "Optional. When normalizing, additionally divides by the sqrt of the "
                 "normalization factor to damp exaggerated features. Default is false."),
    "usessnr": ("BOOL", "Optional. Looks for and uses the class_ssnr header parameter from each "
                "slice to weight each voxel during insertion to the reconstruction."),
    "verbose": ("BOOL", "Optional. Toggles writing useful information to standard out. Default is "
                "false."),
    "quiet": ("BOOL", "Optional. If false, print verbose information."),
    "subvolume": ("INTARRAY", "Optional. (xorigin,yorigin,zorigin,xsize,ysize,zsize) all in "
                  "Fourier pixels. Useful for parallelism."),
    "savenorm": ("STRING", "Debug. Will cause the normalization volume to be written directly to "
                 "the specified file when finish() is called."),
    "normout": ("EMDATA", "Will write the normalization volume to the given EMData object file "
                "when finish() is called."),
}

DESC = ("Reconstruction via direct Fourier methods using one of a variety of different kernels, "
        "most of which are Gaussian based")


def _host_or_device(a):
    """numpy float32 contiguous array, or a contiguous float32 torch tensor as is."""
    if isinstance(a, EMData):
        return a.numpy()
    if hasattr(a, "data_ptr"):
        import torch
        if a.dtype != torch.float32:
            a = a.float()
        return a.contiguous()
    return np.ascontiguousarray(a, np.float32)


def library_stream(handle) -> int:
    """cudaStream_t the handle's work goes to."""
    out = ctypes.c_void_p()
    _lib.check(_lib.load().fr_get_stream(handle, ctypes.byref(out)))
    return out.value or 0


_joins = threading.local()


def _join_parts(ptr: int, dev):
    """This thread's wrapper of library stream `ptr` and its two events,
    reused across calls (a wait takes the event as last recorded, so
    re-recording it later does not move earlier waits)."""
    import torch
    cache = getattr(_joins, "cache", None)
    if cache is None or len(cache) > 256:
        cache = _joins.cache = {}
    key = (ptr, dev.index)
    parts = cache.get(key)
    if parts is None:
        parts = (torch.cuda.ExternalStream(ptr, device=dev), torch.cuda.Event(), torch.cuda.Event())
        cache[key] = parts
    return parts


class join_streams:
    """Around an insertion call given CUDA tensors (the call returns before
    its kernels finish): the library stream first waits for torch's current
    stream, where the tensors were produced, and torch's current stream then
    waits for the library's work, so memory torch frees and hands out again
    is not rewritten before the kernels have read it."""

    def __init__(self, stream_ptr: int, *arrays):
        self.ts = next((a for a in arrays if getattr(a, "is_cuda", False)), None)
        self.ptr = stream_ptr

    def __enter__(self):
        if self.ts is not None:
            import torch
            dev = self.ts.device
            self.cur = torch.cuda.current_stream(dev)
            self.ext, ev_in, self.ev_out = _join_parts(self.ptr, dev)
            ev_in.record(self.cur)
            self.ext.wait_event(ev_in)
        return self

    def __exit__(self, *exc):
        if self.ts is not None:
            self.ev_out.record(self.ext)
            self.cur.wait_event(self.ev_out)
        return False


def _rot_of(xf) -> np.ndarray:
    if isinstance(xf, Transform):
        return xf.rotation_block().astype(np.float32)
    a = np.asarray(xf, np.float32)
    if a.size == 12:
        return np.ascontiguousarray(a.reshape(3, 4)[:, :3])
    return np.ascontiguousarray(a.reshape(3, 3))


def _trans_of(xf):
    if isinstance(xf, Transform):
        return float(xf.matrix[0, 3]), float(xf.matrix[1, 3])
    a = np.asarray(xf, np.float32)
    if a.size == 12:
        m = a.reshape(3, 4)
        return float(m[0, 3]), float(m[1, 3])
    return 0.0, 0.0


class FourierReconstructor:
    """GPU FourierReconstructor with the reference's interface."""

    NAME = "fourier"

    def __init__(self, params: dict | None = None):
        self.params: dict = {}
        self._h = None
        self._sig = None
        self._state = 0
        if params:
            self.insert_params(params)

    # --------------------------------------------------------- factory API
    def get_name(self):
        return self.NAME

    def get_desc(self):
        return DESC

    def get_param_types(self):
        return dict(PARAM_TYPES)

    def get_params(self):
        return dict(self.params)

    def set_params(self, new_params: dict):
        self.params = {}
        self.insert_params(new_params)

    def insert_params(self, new_params: dict):
        """FactoryBase::insert_params (libEM/emobject.h:926-938): unknown key ->
        InvalidParameterException."""
        for k, v in new_params.items():
            if k not in PARAM_TYPES:
                raise InvalidParameterException(k)
            self.params[k] = v

    def set_param(self, key, value):
        self.params[key] = value

    def print_params(self):
        for k, (t, d) in PARAM_TYPES.items():
            print(f"{k}\t{t}\t{d}")

    # --------------------------------------------------------- handle
    @property
    def N(self) -> int:
        return int(self._size()[0])

    @property
    def NZ(self) -> int:
        """The volume's z size (N for the usual cubic volume; a different z
        size, with square N x N slices, takes the scatter insertion)."""
        return int(self._size()[2])

    def _size(self):
        if "size" not in self.params:
            raise NotExistingObjectException("The requested key does not exist: size")
        size = self.params["size"]
        if np.isscalar(size):
            size = [int(size)] * 3
        size = [int(s) for s in size]
        if len(size) != 3:
            raise InvalidParameterException("size must have three elements")
        return size

    def _mode(self) -> str:
        return str(self.params.get("mode", "gauss_2"))

    def _sym(self) -> str:
        return str(self.params.get("sym", "c1"))

    MODE_ID = None   # a fixed inserter (subclasses), else the "mode" parameter's

    def _ensure_handle(self):
        size = self._size()
        mode = self._mode()
        if self.MODE_ID is None and mode not in _lib.MODE_IDS:
            raise UnsupportedParameterException(
                f"mode {mode!r}: the built inserters are {sorted(_lib.MODE_IDS)}")
        if "subvolume" in self.params:
            raise UnsupportedParameterException("subvolume reconstruction is not built")
        sig = (tuple(size), mode, self._sym().lower(), bool(self.params.get("corners", False)),
               bool(self.params.get("sqrtnorm", False)), bool(self.params.get("usessnr", False)))
        if self._h is not None and sig == self._sig:
            return
        self.close()
        lib = _lib.load()
        p = _lib.fr_params()
        p.nx, p.ny, p.nz = size
        p.mode = self.MODE_ID if self.MODE_ID is not None else _lib.MODE_IDS[mode]
        p.sym = self._sym().encode()[:15]
        p.corners = int(sig[3])
        p.sqrtnorm = int(sig[4])
        p.usessnr = int(sig[5])
        p.verbose = int(bool(self.params.get("verbose", False)))
        h = ctypes.c_void_p()
        _lib.check(lib.fr_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self._sig = sig

    def close(self):
        if self._h is not None:
            _lib.load().fr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # --------------------------------------------------------- setup
    def setup(self):
        """FourierReconstructor::setup (libEM/reconstructor.cpp:730-818)."""
        self._ensure_handle()
        _lib.check(_lib.load().fr_setup(self._h))
        self._state = 1

    def setup_seed(self, seed, seed_weight: float):
        """FourierReconstructor::setup_seed (libEM/reconstructor.cpp:820-902)."""
        self._ensure_handle()
        s = _host_or_device(seed)
        N = self.N
        if tuple(s.shape[-3:]) != (N, N, N + 2):
            raise ImageDimensionException(
                "The dimensions of the seed volume do not match the reconstruction size")
        _lib.check(_lib.load().fr_setup_seed(self._h, _lib.ptr(s), float(seed_weight)))
        self._state = 1

    def setup_seedandweights(self, seed, weights):
        """FourierReconstructor::setup_seedandweights (libEM/reconstructor.cpp:904-996)."""
        self._ensure_handle()
        s, w = _host_or_device(seed), _host_or_device(weights)
        N = self.N
        if tuple(s.shape[-3:]) != (N, N, N + 2) or tuple(w.shape[-3:]) != (N, N, N // 2 + 1):
            raise ImageDimensionException(
                "The dimensions of the seed volume do not match the reconstruction size")
        _lib.check(_lib.load().fr_setup_seedandweights(self._h, _lib.ptr(s), _lib.ptr(w)))
        self._state = 1

    def clear(self):
        _lib.check(_lib.load().fr_clear(self._h))

    # --------------------------------------------------------- slices
    def _check_image(self, a, complex_: bool):
        N = self.N
        want = (N, N + 2) if complex_ else (N, N)
        if tuple(a.shape[-2:]) != want:
            raise ImageDimensionException(
                f"slice is {tuple(a.shape[-2:])}, expected {want} for a {N}^3 reconstruction")

    def preprocess_slice(self, img, xform) -> EMData:
        """FourierReconstructor::preprocess_slice (libEM/reconstructor.cpp:1022-1061):
        translation (bilinear), phase origin to corner, r2c, x sqrt((N+2)/N)."""
        if img is None:
            raise NullPointerException("EMData pointer (input image) is NULL")
        self._ensure_handle()
        a = _host_or_device(img)
        self._check_image(a, False)
        tx, ty = _trans_of(xform if xform is not None else Transform())
        inv = np.array([-tx, -ty], np.float32)   # the xform processor applies t^-1
        N = self.N
        out = np.empty((N, N + 2), np.float32)
        _lib.check(_lib.load().fr_preprocess_slices(self._h, _lib.ptr(a), 1, _lib.ptr(inv),
                                                    _lib.ptr(out)))
        res = EMData(out, is_complex=True,
                     attrs=dict(img.attrs) if isinstance(img, EMData) else None)
        res.set_attr("reconstruct_preproc", 1)
        return res

    def _slice_of(self, img, xform):
        if isinstance(img, EMData) and img.get_attr_default("reconstruct_preproc", 0):
            a = img.numpy()
            self._check_image(a, True)
            return a
        if isinstance(img, EMData) and img.is_complex():
            a = img.numpy()
            self._check_image(a, True)
            return a
        return self.preprocess_slice(img, xform).numpy()

    def insert_slice(self, img, xform, weight: float = 1.0) -> int:
        """FourierReconstructor::insert_slice (libEM/reconstructor.cpp:1064-1119).
        Returns 0, or -1 when the weight is 0 (nothing inserted).  One slice per
        call: the plain per-call GPU path."""
        if img is None:
            raise NullPointerException("EMData pointer (input image) is NULL")
        if self._state != 1:
            self._require_setup()
        usessnr = bool(self.params.get("usessnr", False))
        ssnr = None
        if isinstance(img, EMData) and img.has_attr("class_ssnr"):
            ssnr = np.ascontiguousarray(img.get_attr("class_ssnr"), np.float32)
        if usessnr:
            weight = -1.0 if ssnr is not None else 0.0
        if float(weight) == 0.0:
            return -1
        if float(weight) < 0.0 and ssnr is None:
            # the SSNR path reads class_ssnr (libEM/reconstructor.cpp:1160-1162)
            raise NotExistingObjectException("The requested key does not exist: class_ssnr")
        if float(weight) > 0.0:
            ssnr = None
        sl = self._slice_of(img, xform)
        rot = _rot_of(xform)
        w = np.array([weight], np.float32)
        status = (ctypes.c_int * 1)()
        _lib.check(_lib.load().fr_insert_slices(
            self._h, _lib.ptr(sl), 1, _lib.ptr(rot), _lib.ptr(w),
            _lib.ptr(ssnr) if ssnr is not None else None,
            int(ssnr.size) if ssnr is not None else 0, status, _lib.SCHED["scatter"]))
        return int(status[0])

    def insert_slices(self, slices, rots, weights, schedule: str = "auto"):
        """Batched insert_slice over n preprocessed slices (n, N, N+2) with
        rotation blocks (n, 3, 3) and weights (n,).  Returns the per-slice
        insert_slice return values."""
        if self._state != 1:
            self._require_setup()
        s = _host_or_device(slices)
        self._check_image(s, True)
        n = int(s.shape[0]) if s.ndim == 3 else 1
        r = _host_or_device(rots)
        w = _host_or_device(weights)
        status = (ctypes.c_int * n)()
        with join_streams(library_stream(self._h), s, r, w):
            _lib.check(_lib.load().fr_insert_slices(self._h, _lib.ptr(s), n, _lib.ptr(r), _lib.ptr(w),
                                                    None, 0, status, _lib.SCHED[schedule]))
        return list(status)

    def insert_particles(self, images, meta, schedule: str = "auto"):
        """The reference caller's per-particle loop (programs/e2spa_make3d.py:300-345)
        for n raw box x box particles: edge-mean subtract, clip to N, CTF phase
        flip, edge-mean subtract, shift, preprocess, insert.  ``meta`` is an
        array of ``_lib.fr_particle`` (see ``eman2_b200.particles``)."""
        if self._state != 1:
            self._require_setup()
        a = _host_or_device(images)
        n, box = int(a.shape[0]), int(a.shape[-1])
        with join_streams(library_stream(self._h), a):
            _lib.check(_lib.load().fr_insert_particles(self._h, _lib.ptr(a), n, box,
                                                       ctypes.cast(meta, ctypes.c_void_p),
                                                       _lib.SCHED[schedule]))

    def determine_slice_agreement(self, img, xform, weight: float = 1.0, sub: bool = True) -> int:
        """FourierReconstructor::determine_slice_agreement
        (libEM/reconstructor.cpp:1212-1257).  Sets reconstruct_norm,
        reconstruct_absqual, reconstruct_absqual_lowres and reconstruct_weight
        on ``img``; returns 0."""
        if img is None:
            raise NullPointerException("EMData pointer (input image) is NULL")
        if self._state != 1:
            self._require_setup()
        sl = self._slice_of(img, xform)
        rot = _rot_of(xform)
        w = np.array([weight], np.float32)
        apix = float(img.get_attr_default("apix_x", 1.0)) if isinstance(img, EMData) else 1.0
        out = np.zeros(5, np.float32)
        _lib.check(_lib.load().fr_determine_slice_agreement(
            self._h, _lib.ptr(sl), 1, _lib.ptr(rot), _lib.ptr(w), apix, int(bool(sub)),
            _lib.ptr(out)))
        if isinstance(img, EMData):
            img.set_attr("reconstruct_norm", float(out[0]))
            img.set_attr("reconstruct_absqual", float(out[1]))
            img.set_attr("reconstruct_absqual_lowres", float(out[2]))
            img.set_attr("reconstruct_weight", float(out[4]))
        return 0

    def slice_agreement(self, slices, rots, weights, apix: float = 1.0) -> np.ndarray:
        """Batched determine_slice_agreement(sub=False): (n, 5) array of
        reconstruct_norm, _absqual, _absqual_lowres, _qual, _weight."""
        s = _host_or_device(slices)
        n = int(s.shape[0]) if s.ndim == 3 else 1
        r = _host_or_device(rots)
        w = _host_or_device(weights)
        out = np.zeros((n, 5), np.float32)
        _lib.check(_lib.load().fr_determine_slice_agreement(
            self._h, _lib.ptr(s), n, _lib.ptr(r), _lib.ptr(w), float(apix), 0, _lib.ptr(out)))
        return out

    def projection(self, xform, ret_fourier: int = 1) -> EMData:
        """FourierReconstructor::projection (libEM/reconstructor.cpp:1383-1445)
        of the current accumulators: the slice through the volume at the
        transform's rotation, shifted by its translation; ret_fourier=1 the
        complex slice (N, N+2), 0 the real (N, N) image (phase origin to the
        centre, inverse FFT)."""
        if self._state != 1:
            self._require_setup()
        N = self.N
        xf = np.zeros((3, 4), np.float32)
        xf[:, :3] = _rot_of(xform)
        xf[0, 3], xf[1, 3] = _trans_of(xform)
        out = np.zeros((N, N + 2) if ret_fourier else (N, N), np.float32)
        _lib.check(_lib.load().fr_projection_xf(self._h, _lib.ptr(xf), int(bool(ret_fourier)),
                                                _lib.ptr(out)))
        return EMData(out, is_complex=bool(ret_fourier))

    # --------------------------------------------------------- results
    def get_accumulators(self):
        """Un-normalised (complex, weight) volumes: what finish(False) + normout
        give before normalisation."""
        N, NZ = self.N, self.NZ
        d = np.empty((NZ, N, N + 2), np.float32)
        n = np.empty((NZ, N, N // 2 + 1), np.float32)
        _lib.check(_lib.load().fr_get_accumulators(self._h, _lib.ptr(d), _lib.ptr(n)))
        return d, n

    def finish(self, doift: bool = True) -> EMData:
        """FourierReconstructor::finish (libEM/reconstructor.cpp:1552-1641).
        doift: real N^3 map (phase origin at the centre); else the normalised
        complex volume.  Fills the ``normout`` EMData if that param is set."""
        if self._state != 1:
            self._require_setup()
        N, NZ = self.N, self.NZ
        out = np.empty((NZ, N, N) if doift else (NZ, N, N + 2), np.float32)
        norm = np.empty((NZ, N, N // 2 + 1), np.float32)
        _lib.check(_lib.load().fr_finish(self._h, int(bool(doift)), _lib.ptr(out), _lib.ptr(norm)))
        self._state = 2
        if "normout" in self.params and isinstance(self.params["normout"], EMData):
            self.params["normout"].set_data(norm)
        if self.params.get("savenorm"):
            np.save(str(self.params["savenorm"]), norm)
        return EMData(out, is_complex=not doift)

    def finish_async(self, doift: bool = True, stream=None) -> "PendingFinish":
        """finish() enqueued without waiting (fr_finish_async): the map and
        the weights are written into page-locked host buffers on ``stream``
        (a torch CUDA stream; default the library stream).  Returns a
        PendingFinish: ready() polls, result() waits and returns the EMData
        (and fills the ``normout`` EMData, as finish() does)."""
        import torch
        if self._state != 1:
            self._require_setup()
        N, NZ = self.N, self.NZ
        out = torch.empty((NZ, N, N) if doift else (NZ, N, N + 2), dtype=torch.float32,
                          pin_memory=True)
        norm = torch.empty((NZ, N, N // 2 + 1), dtype=torch.float32, pin_memory=True)
        if stream is None:
            dev = torch.device("cuda", torch.cuda.current_device())
            stream = _join_parts(library_stream(self._h), dev)[0]
        _lib.check(_lib.load().fr_finish_async(self._h, int(bool(doift)), out.data_ptr(),
                                               norm.data_ptr(), ctypes.c_void_p(stream.cuda_stream)))
        ev = torch.cuda.Event()
        ev.record(stream)
        self._state = 2
        return PendingFinish(self, out, norm, ev, not doift)

    # e2make3dpar's Gaussian widths per mode (programs/e2make3dpar.py:422)
    KERNEL_FIX_WIDTH = {"gauss_2": 4.0, "gauss_3": 6.4, "gauss_4": 8.8, "gauss_5": 10.4,
                        "gauss_5_slow": 10.4}

    def finish_corrected(self, gauss_width: float | None = None, outsize=None) -> EMData:
        """finish(True) plus what e2make3dpar does next (programs/e2make3dpar.py:421-431):
        math.gausskernelfix with the mode's Gaussian width (or ``gauss_width``;
        0 or a mode without one: no correction) and the clip to ``outsize``
        (an int or (x, y, z); default N), fused into the pass that writes the
        real map."""
        if self._state != 1:
            self._require_setup()
        N = self.N
        if gauss_width is None:
            gauss_width = self.KERNEL_FIX_WIDTH.get(self.params.get("mode", "gauss_2"), 0.0)
        if outsize is None:
            outsize = (N, N, N)
        elif np.isscalar(outsize):
            outsize = (int(outsize),) * 3
        ox, oy, oz = (int(v) for v in outsize)
        out = np.empty((oz, oy, ox), np.float32)
        norm = np.empty((N, N, N // 2 + 1), np.float32)
        _lib.check(_lib.load().fr_finish_corrected(self._h, float(gauss_width), ox, oy, oz,
                                                   _lib.ptr(out), _lib.ptr(norm)))
        self._state = 2
        if "normout" in self.params and isinstance(self.params["normout"], EMData):
            self.params["normout"].set_data(norm)
        if self.params.get("savenorm"):
            np.save(str(self.params["savenorm"]), norm)
        return EMData(out)

    def _require_setup(self):
        raise StateException("setup() has not been called" if self._state == 0 else
                             "finish() was called; call setup() again")


class PendingFinish:
    """A finish enqueued by FourierReconstructor.finish_async."""

    def __init__(self, owner, out, norm, event, is_complex):
        self.owner = owner
        self._out, self._norm, self._event = out, norm, event
        self._complex = is_complex
        self._result = None

    def ready(self) -> bool:
        return self._result is not None or self._event.query()

    def result(self) -> EMData:
        if self._result is None:
            self._event.synchronize()
            r = self.owner
            if "normout" in r.params and isinstance(r.params["normout"], EMData):
                r.params["normout"].set_data(self._norm.numpy().copy())
            self._result = EMData(self._out.numpy().copy(), is_complex=self._complex)
            self._out = self._norm = None
        return self._result


class WienerFourierReconstructor(FourierReconstructor):
    """WienerFourierReconstructor ("wiener_fourier", libEM/reconstructor.cpp:1643-1731,
    1921-1947): each slice's pixels are weighted by its ctf_snr_total curve at
    the pixel's radius (inside the rn < 0.5 disk) and finish divides by the
    summed weight plus one (a Wiener filter)."""

    NAME = "wiener_fourier"

    def _ensure_handle(self):
        super()._ensure_handle()
        _lib.check(_lib.load().fr_set_wiener(self._h, 1))

    def insert_slice(self, img, xform, weight: float = 1.0) -> int:
        """WienerFourierReconstructor::insert_slice: requires the slice's
        ctf_snr_total; ctf_wiener_filtered undoes a Wiener filter; a negative
        weight subtracts.  Returns 0."""
        if img is None:
            raise NullPointerException("EMData pointer (input image) is NULL")
        if self._state != 1:
            self._require_setup()
        if not (isinstance(img, EMData) and img.has_attr("ctf_snr_total")):
            raise NotExistingObjectException(
                "ctf_snr_total: No SNR information present in class-average. Must use the "
                "ctf.auto or ctfw.auto averager.")
        snr = np.ascontiguousarray(img.get_attr("ctf_snr_total"), np.float32)
        undo = np.array([int(img.get_attr_default("ctf_wiener_filtered", 0))], np.int32)
        sl = self._slice_of(img, xform)
        rot = _rot_of(xform)
        w = np.array([weight], np.float32)
        status = (ctypes.c_int * 1)()
        _lib.check(_lib.load().fr_insert_slices_wiener(
            self._h, _lib.ptr(sl), 1, _lib.ptr(rot), _lib.ptr(w), _lib.ptr(snr), int(snr.size),
            _lib.ptr(undo), status))
        return 0

    def insert_slices_wiener(self, slices, rots, weights, snr, undo=None):
        """n preprocessed slices with their SNR curves snr (n, nsnr)."""
        if self._state != 1:
            self._require_setup()
        s = _host_or_device(slices)
        n = int(s.shape[0])
        r, w = _host_or_device(rots), _host_or_device(weights)
        c = np.ascontiguousarray(snr, np.float32).reshape(n, -1)
        u = np.zeros(n, np.int32) if undo is None else np.ascontiguousarray(undo, np.int32)
        _lib.check(_lib.load().fr_insert_slices_wiener(
            self._h, _lib.ptr(s), n, _lib.ptr(r), _lib.ptr(w), _lib.ptr(c), int(c.shape[1]),
            _lib.ptr(u), None))

    def determine_slice_agreement(self, img, xform, weight: float = 1.0, sub: bool = True) -> int:
        raise UnsupportedParameterException(
            "determine_slice_agreement of wiener_fourier is not built")


class FourierIterReconstructor(FourierReconstructor):
    """FourierIterReconstructor ("fourier_iter", libEM/reconstructor.cpp:430-682):
    a gauss_5-shaped window whose width grows with resolution on the first
    pass; given a seed (the previous iteration's map) it inserts the update
    dt + ref(i,j,k) - ref(p) with a fixed width instead.  finish() normalises
    without sqrtnorm; determine_slice_agreement does nothing and returns 0."""

    NAME = "fourier_iter"
    MODE_ID = _lib.MODE_ITER

    def _ensure_handle(self):
        self.params.pop("sqrtnorm", None)            # finish uses normalize_threed(0)
        super()._ensure_handle()

    def setup_seed(self, seed, seed_weight: float = 1.0):
        """FourierIterReconstructor::setup_seed (:481-488): setup(), then the
        seed (a real N^3 map, or its complex transform) as the reference."""
        self.setup()
        s = _host_or_device(seed.numpy() if isinstance(seed, EMData) else seed)
        N = self.N
        is_complex = tuple(s.shape[-3:]) == (N, N, N + 2)
        if not is_complex and tuple(s.shape[-3:]) != (N, N, N):
            raise ImageDimensionException(
                "The dimensions of the seed volume do not match the reconstruction size")
        with join_streams(library_stream(self._h), s):
            _lib.check(_lib.load().fr_set_reference(self._h, _lib.ptr(s), int(is_complex)))

    def setup_seedandweights(self, seed, weights):
        """The weights are ignored, as in the reference (:490-499)."""
        self.setup_seed(seed)

    def clear(self):
        """FourierIterReconstructor::clear (:501-503): setup() again."""
        self.setup()

    def insert_slice(self, img, xform, weight: float = 1.0) -> int:
        """FourierIterReconstructor::insert_slice (:522-648).  Returns 0."""
        if img is None:
            raise NullPointerException("EMData pointer (input image) is NULL")
        if self._state != 1:
            self._require_setup()
        sl = self._slice_of(img, xform)
        rot = _rot_of(xform)
        w = np.array([weight], np.float32)
        status = (ctypes.c_int * 1)()
        _lib.check(_lib.load().fr_insert_slices(self._h, _lib.ptr(sl), 1, _lib.ptr(rot), _lib.ptr(w),
                                                None, 0, status, _lib.SCHED["scatter"]))
        return 0

    def determine_slice_agreement(self, img, xform, weight: float = 1.0, sub: bool = True) -> int:
        return 0


class Reconstructors:
    """Factory<Reconstructor> (libpyEM/libpyReconstructor2.cpp:221-226)."""

    _known = {"fourier": FourierReconstructor, "wiener_fourier": WienerFourierReconstructor,
              "fourier_iter": FourierIterReconstructor}

    @staticmethod
    def get(name: str, params: dict | None = None):
        cls = Reconstructors._known.get(name)
        if cls is None:
            raise NotExistingObjectException(f"No such an instance existing: {name}")
        return cls(params)

    @staticmethod
    def get_list():
        return list(Reconstructors._known)
