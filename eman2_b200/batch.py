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

import numpy as np

from . import _lib
from .emdata import EMData
from .reconstructor import FourierReconstructor, _host_or_device, join_streams, library_stream


def insert_particles_multi(recons, images, metas, stream=None):
    """One batched insertion tick over already set-up reconstructions:
    images[j] (n_j, box_j, box_j) and metas[j] (fr_particle array) go to
    recons[j]."""
    nj = len(recons)
    lib = _lib.load()
    keep = [_host_or_device(im) for im in images]
    handles = (ctypes.c_void_p * nj)(*[r.handle.value for r in recons])
    imgs = (ctypes.c_void_p * nj)(*[_lib.ptr(a) for a in keep])
    boxes = (ctypes.c_int * nj)(*[int(a.shape[-1]) for a in keep])
    counts = (ctypes.c_int * nj)(*[int(a.shape[0]) for a in keep])
    metas_p = (ctypes.c_void_p * nj)(*[ctypes.cast(m, ctypes.c_void_p).value for m in metas])
    st = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
    with join_streams(st.value if st is not None else library_stream(recons[0].handle), *keep):
        _lib.check(lib.fr_insert_particles_multi(handles, nj, imgs, boxes, counts, metas_p, st))


TILE_NAMES = {0: "gather 8x8x8", 1: "gather 16x8x8", 2: "gather 8x8x4", 3: "gather 16x16x4",
              4: "column (staged)", 5: "column (barrier-free)", -2: "scatter"}


def autotune(N: int, mode: str, nsym: int, nparticles: int = 256):
    """Times every insertion schedule for (N, mode, nsym) on random slices and
    records the fastest; batched and plain insertions of that shape use it
    from then on.  Returns (tile id, {schedule name: ms})."""
    lib = _lib.load()
    tile = ctypes.c_int()
    ms = (ctypes.c_float * 7)()
    _lib.check(lib.fr_autotune(int(N), _lib.MODE_IDS[mode], int(nsym), int(nparticles),
                               ctypes.byref(tile), ms))
    names = [TILE_NAMES[i] for i in range(6)] + [TILE_NAMES[-2]]
    return tile.value, dict(zip(names, list(ms)))


def set_tile(N: int, mode: str, nsym: int, tile: int):
    """Pins the schedule for (N, mode, nsym) (tile ids as TILE_NAMES; -1 clears)."""
    _lib.check(_lib.load().fr_set_tile(int(N), _lib.MODE_IDS[mode], int(nsym), int(tile)))


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

    def get_accumulators(self, j: int):
        return self.recons[j].get_accumulators()

    def finish(self, j: int, doift: bool = True) -> EMData:
        return self.recons[j].finish(doift)

    def close(self):
        for r in self.recons:
            r.close()
