"""Batched form: many independent reconstructions (uneven box sizes, modes,
symmetries -- even/odd half maps, heterogeneity classes) inserted by one
persistent insertion launch per round of particle chunks.

The arithmetic is the plain path's: each job gets exactly the taps
``FourierReconstructor.insert_particles`` would give it; only the execution
(one launch over every job's (voxel tile, slice block) work items, heaviest
first) changes.
"""
from __future__ import annotations

import ctypes
import sys

import numpy as np

from . import _lib
from .emdata import EMData
from .reconstructor import FourierReconstructor, _host_or_device, join_streams, library_stream


def _meta_address(m):
    """Address of an fr_particle array (or pointer); None stays None."""
    if m is None:
        return None
    if isinstance(m, ctypes.Array):
        return ctypes.addressof(m)
    return ctypes.cast(m, ctypes.c_void_p).value


def _particles(images):
    """Particle arrays of a batched call as the library reads them, and their
    addresses.  Contiguous float32 tensors pass through untouched: the common
    case, kept cheap since a call converts one array per job."""
    torch = sys.modules.get("torch")
    keep, ptrs = [], []
    for a in images:
        if a is None:
            keep.append(None)
            ptrs.append(None)
        elif torch is not None and isinstance(a, torch.Tensor) and a.dtype is torch.float32 \
                and a.is_contiguous():
            keep.append(a)
            ptrs.append(a.data_ptr())
        else:
            a = _host_or_device(a)
            keep.append(a)
            ptrs.append(_lib.ptr(a))
    return keep, ptrs


def insert_particles_multi(recons, images, metas, stream=None):
    """One batched insertion tick over already set-up reconstructions:
    images[j] (n_j, box_j, box_j) and metas[j] (fr_particle array) go to
    recons[j]."""
    nj = len(recons)
    lib = _lib.load()
    keep, ptrs = _particles(images)
    handles = (ctypes.c_void_p * nj)(*[r.handle.value for r in recons])
    imgs = (ctypes.c_void_p * nj)(*ptrs)
    boxes = (ctypes.c_int * nj)(*[int(a.shape[-1]) for a in keep])
    counts = (ctypes.c_int * nj)(*[int(a.shape[0]) for a in keep])
    metas_p = (ctypes.c_void_p * nj)(*[_meta_address(m) for m in metas])
    st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
    with join_streams(st.value if st is not None else library_stream(recons[0].handle), *keep):
        _lib.check(lib.fr_insert_particles_multi(handles, nj, imgs, boxes, counts, metas_p, st))


TILE_NAMES = {0: "gather 8x8x8", 1: "gather 16x8x8", 2: "gather 8x8x4", 3: "gather 16x16x4",
              4: "column (staged)", 5: "column (barrier-free)", 6: "pixel-major", -2: "scatter"}


def autotune(N: int, mode: str, nsym: int, nparticles: int = 256):
    """Times every insertion schedule for (N, mode, nsym) on random slices and
    records the fastest; batched and plain insertions of that shape use it
    from then on.  Returns (tile id, {schedule name: ms})."""
    lib = _lib.load()
    tile = ctypes.c_int()
    ms = (ctypes.c_float * 8)()
    _lib.check(lib.fr_autotune(int(N), _lib.MODE_IDS[mode], int(nsym), int(nparticles),
                               ctypes.byref(tile), ms))
    names = [TILE_NAMES[i] for i in range(7)] + [TILE_NAMES[-2]]
    return tile.value, dict(zip(names, list(ms)))


def set_tile(N: int, mode: str, nsym: int, tile: int):
    """Pins the schedule for (N, mode, nsym) (tile ids as TILE_NAMES; -1 clears)."""
    _lib.check(_lib.load().fr_set_tile(int(N), _lib.MODE_IDS[mode], int(nsym), int(tile)))


class InsertGraph:
    """A batched insertion round of fixed shapes captured once as a CUDA graph
    (fr_graph_create): every replay inserts counts[j] particles of box
    boxes[j] into recons[j] through the same prologue and persistent launches
    as insert_particles_multi, without per-round host work beyond staging
    the particles' metadata and image addresses.  ctf[j]: whether job j's
    particles carry a CTF (replays with CTF particles need it set for a job of
    the same N, box and symmetry)."""

    def __init__(self, recons, boxes, counts, ctf, stream=None):
        lib = _lib.load()
        self.recons = list(recons)
        nj = len(self.recons)
        self.boxes, self.counts = [int(b) for b in boxes], [int(c) for c in counts]
        handles = (ctypes.c_void_p * nj)(*[r.handle.value for r in self.recons])
        cb = (ctypes.c_int * nj)(*self.boxes)
        cc = (ctypes.c_int * nj)(*self.counts)
        cf = (ctypes.c_int * nj)(*[1 if c else 0 for c in ctf])
        self.stream_ptr = stream.cuda_stream if stream is not None else \
            library_stream(self.recons[0].handle)
        out = ctypes.c_void_p()
        _lib.check(lib.fr_graph_create(handles, nj, cb, cc, cf, ctypes.c_void_p(self.stream_ptr),
                                       ctypes.byref(out)))
        self._g = out

    def slot(self, j: int) -> int:
        """Device address of job j's image slot, float[counts[j]][box][box]."""
        p = ctypes.c_void_p()
        _lib.check(_lib.load().fr_graph_slot(self._g, int(j), ctypes.byref(p)))
        return p.value

    def launch(self, images, metas):
        """One replay.  images[j]: (counts[j], box, box) host particles (copied
        into the slots) or device particles (read in place), or None to insert
        what the slots hold; metas[j]: fr_particle arrays of counts[j] entries."""
        nj = len(self.recons)
        metas_p = (ctypes.c_void_p * nj)(*[_meta_address(m) for m in metas])
        if images is None:
            _lib.check(_lib.load().fr_graph_launch(self._g, None, metas_p))
            return
        keep, ptrs = _particles(images)
        imgs = (ctypes.c_void_p * nj)(*ptrs)
        with join_streams(self.stream_ptr, *[a for a in keep if a is not None]):
            _lib.check(_lib.load().fr_graph_launch(self._g, imgs, metas_p))

    def close(self):
        if getattr(self, "_g", None):
            _lib.check(_lib.load().fr_graph_destroy(self._g))
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchReconstructor:
    """A fixed set of reconstructions inserted together (fr_batch_*)."""

    def __init__(self, jobs: list[dict]):
        self.recons = []
        for p in jobs:
            r = FourierReconstructor(p)
            r.setup()
            self.recons.append(r)

    def __len__(self):
        return len(self.recons)

    def insert_particles(self, images: list, metas: list, stream=None):
        """images[j]: (n_j, box_j, box_j) raw particles of job j (n_j may be 0
        for a job with nothing this round); metas[j]: its fr_particle array."""
        active = [j for j in range(len(self.recons)) if int(np.shape(images[j])[0]) > 0]
        if not active:
            return
        insert_particles_multi([self.recons[j] for j in active], [images[j] for j in active],
                               [metas[j] for j in active], stream)

    def capture(self, boxes, counts, ctf, stream=None) -> InsertGraph:
        """A CUDA graph of one insertion round of these shapes (InsertGraph)."""
        return InsertGraph(self.recons, boxes, counts, ctf, stream)

    def get_accumulators(self, j: int):
        return self.recons[j].get_accumulators()

    def finish(self, j: int, doift: bool = True) -> EMData:
        return self.recons[j].finish(doift)

    def close(self):
        for r in self.recons:
            r.close()
