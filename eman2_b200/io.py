"""Particle I/O feeding the reconstruction: MRC images and stacks
(libEM/io/mrcio.cpp), EMAN2's fast LST particle lists (#LSX,
libEM/io/lstfastio.cpp, libpyEM/EMAN2.py LSXFile) and a reader that streams
particle chunks from disk into HBM while earlier chunks are inserted.

Stacks move in their stored width: a chunk's raw bytes are read straight
into pinned host memory, copied to the device undecoded and widened to
float32 there (fr_decode_images), so a 16-bit stack crosses PCIe at half the
bytes of its float32 image.
"""
from __future__ import annotations

import ctypes
import json
import os
import threading

import numpy as np

from . import _lib
from .emdata import EMData
from .exceptions import ImageDimensionException, NotExistingObjectException
from .transform import Transform

# ------------------------------------------------------------------ MRC

HEADER_BYTES = 1024
# MrcIO::MrcMode (libEM/io/mrcio.h:63-74) and the element each mode stores;
# mode 0 is read as unsigned bytes, as MrcIO::read_data does.
MODE_DTYPE = {0: np.uint8, 17: np.int8, 1: np.int16, 6: np.uint16, 12: np.float16,
              2: np.float32}
MODE_BITS = {0: 8, 17: 8, 1: 16, 6: 16, 12: 16, 2: 32, 101: 4}


class MrcInfo:
    """Header fields the reader needs (word offsets as MrcHeader,
    libEM/io/mrcio.h:87-160)."""

    def __init__(self, path: str, words: np.ndarray, fwords: np.ndarray, swap: bool):
        self.path = path
        self.nx, self.ny, self.nz, self.mode = (int(v) for v in words[:4])
        self.mx, self.my, self.mz = (int(v) for v in words[7:10])
        self.xlen, self.ylen, self.zlen = (float(v) for v in fwords[10:13])
        self.nsymbt = int(words[23])
        self.swap = swap
        ext = os.path.splitext(path)[1].lower()
        self.is_stack = ext == ".mrcs"                    # MrcIO::init (mrcio.cpp:117)
        self.nimg = self.nz if self.is_stack else 1
        self.data_offset = HEADER_BYTES + self.nsymbt     # mrcio.cpp:1054
        self.apix = self.xlen / self.mx if self.mx > 0 and self.xlen > 0 else 1.0
        if self.mode not in MODE_BITS:
            raise ImageDimensionException(f"{path}: MRC mode {self.mode} is not supported")

    @property
    def image_values(self) -> int:
        return self.nx * self.ny * (1 if self.is_stack else self.nz)

    @property
    def image_bytes(self) -> int:
        return self.image_values * MODE_BITS[self.mode] // 8


def _plausible(w) -> bool:
    nx, ny, nz, mode = (int(v) for v in w[:4])
    return 0 < nx < 1 << 20 and 0 < ny < 1 << 20 and 0 < nz < 1 << 24 and mode in MODE_BITS


def mrc_info(path: str) -> MrcInfo:
    """Reads and byte-order-checks an MRC header.  The order is the one the
    machine stamp names (0x44 0x44 / 0x44 0x41 little, 0x11 0x11 big), else
    the one under which nx, ny, nz and mode are plausible (the role of
    MrcIO::check_swap, libEM/io/mrcio.cpp:234-340)."""
    with open(path, "rb") as f:
        hdr = f.read(HEADER_BYTES)
    if len(hdr) < HEADER_BYTES:
        raise NotExistingObjectException(f"{path}: not an MRC file (short header)")
    stamp = hdr[212:214]
    le = np.frombuffer(hdr, "<i4"), np.frombuffer(hdr, "<f4")
    be = np.frombuffer(hdr, ">i4"), np.frombuffer(hdr, ">f4")
    if stamp in (b"\x44\x44", b"\x44\x41") and _plausible(le[0]):
        w, swap = le, False
    elif stamp == b"\x11\x11" and _plausible(be[0]):
        w, swap = be, True
    elif _plausible(le[0]):
        w, swap = le, False
    elif _plausible(be[0]):
        w, swap = be, True
    else:
        raise NotExistingObjectException(f"{path}: not an MRC file")
    return MrcInfo(path, w[0], w[1], swap)


def _decode_host(raw: np.ndarray, info: MrcInfo) -> np.ndarray:
    if info.mode == 101:
        b = raw.view(np.uint8)
        out = np.empty(b.size * 2, np.float32)
        out[0::2] = b & 15
        out[1::2] = b >> 4
        return out
    dt = np.dtype(MODE_DTYPE[info.mode]).newbyteorder(">" if info.swap else "<")
    return raw.view(dt).astype(np.float32)


def read_mrc(path: str, index: int = 0) -> EMData:
    """EMData(path, index): image `index` of a .mrcs stack, else the whole map."""
    info = mrc_info(path)
    if index != 0 and not info.is_stack:
        raise ImageDimensionException("no stack allowed for MRC image")
    if not 0 <= index < info.nimg:
        raise ImageDimensionException(f"{path}: image {index} of {info.nimg}")
    with open(path, "rb") as f:
        f.seek(info.data_offset + index * info.image_bytes)
        raw = np.frombuffer(f.read(info.image_bytes), np.uint8)
    a = _decode_host(raw, info)
    shape = (info.ny, info.nx) if info.is_stack or info.nz == 1 else (info.nz, info.ny, info.nx)
    e = EMData(a.reshape(shape))
    e.set_attr("apix_x", info.apix)
    e.set_attr("apix_y", info.apix)
    e.set_attr("apix_z", info.apix)
    return e


def read_mrc_stack(path: str, first: int = 0, n: int | None = None) -> np.ndarray:
    """Images first..first+n of a .mrcs stack as float32 (n, ny, nx)."""
    info = mrc_info(path)
    n = info.nimg - first if n is None else n
    raw = np.fromfile(path, np.uint8, count=n * info.image_bytes,
                      offset=info.data_offset + first * info.image_bytes)
    return _decode_host(raw, info).reshape(n, info.ny, info.nx)


def write_mrc(path: str, data, apix: float = 1.0, mode: int = 2):
    """Writes a float32 image, volume or (for a .mrcs path) stack, little
    endian, in mode 2 (float32), 12 (float16) or 1 (int16, values rounded)."""
    a = np.ascontiguousarray(np.asarray(data, np.float32))
    if a.ndim == 2:
        a = a[None]
    nz, ny, nx = a.shape
    stack = os.path.splitext(path)[1].lower() == ".mrcs"
    store = {2: np.float32, 12: np.float16, 1: np.int16}[mode]
    body = (np.rint(a) if mode == 1 else a).astype(store).astype(np.dtype(store).newbyteorder("<"))
    hdr = np.zeros(256, "<i4")
    fh = hdr.view("<f4")
    hdr[0:4] = nx, ny, nz, mode
    hdr[7:10] = nx, ny, (1 if stack else nz)
    fh[10:13] = nx * apix, ny * apix, (1 if stack else nz) * apix
    fh[13:16] = 90.0
    hdr[16:19] = 1, 2, 3
    fh[19], fh[20], fh[21] = float(a.min()), float(a.max()), float(a.mean())
    hdr[22] = 0 if (stack or nz == 1) else 1              # ispg: images 0, volume 1
    hdr[23] = 0
    hdr[27] = 20140                                       # nversion (MRC2014)
    raw = bytearray(hdr.tobytes())
    raw[208:212] = b"MAP "
    raw[212:216] = b"\x44\x44\x00\x00"
    raw[216:220] = np.float32(a.std()).tobytes()          # rms
    raw[220:224] = np.int32(1).tobytes()
    label = b"eman2_b200"
    raw[224:224 + len(label)] = label
    with open(path, "wb") as f:
        f.write(bytes(raw))
        f.write(body.tobytes())


# ------------------------------------------------------------------ LSX

def _json_to_obj(d):
    """EMAN2jsondb.json_to_obj for the classes particle lists carry
    (libpyEM/EMAN2jsondb.py:942-961, Transform :192-208)."""
    if d.get("__class__") == "Transform":
        m = d["matrix"]
        if isinstance(m, str):
            m = [float(v) for v in m[1:-1].split(",")]
        return Transform(m)
    return d


def _obj_to_json(o):
    if isinstance(o, Transform):
        # Transform::get_matrix_string(6) (libEM/transform.cpp:169-178)
        return {"__class__": "Transform",
                "matrix": "[" + ",".join("%1.6g" % v for v in o.get_matrix()) + "]"}
    if isinstance(o, np.ndarray):
        return o.tolist()
    if isinstance(o, np.generic):
        return o.item()
    raise TypeError(f"not JSON serialisable: {type(o)}")


class LSXFile:
    """EMAN2's fast LST file (libpyEM/EMAN2.py LSXFile, libEM/io/lstfastio.cpp):
    '#LSX', a comment line, '# <line length>', then fixed-length records
    '<n in file>\\t<image file>[\\t<JSON dict>]' padded with spaces."""

    COMMENT = ("# This file is in fast LST format. All lines after the next line have exactly "
               "the number of characters shown on the next line. This MUST be preserved if editing.")

    def __init__(self, path: str, ifexists: bool = False, comments: str = ""):
        self.path = path
        if not os.path.exists(path):
            if ifexists:
                raise NotExistingObjectException(f"lst file {path} does not exist")
            with open(path, "w") as f:
                f.write("#LSX\n{}\n# 20\n".format(comments or self.COMMENT))
        self.ptr = open(path, "r+")
        if self.ptr.readline() != "#LSX\n":
            raise NotExistingObjectException(f"{path} is not in #LSX format")
        self.filecomment = self.ptr.readline().strip()
        self.linelen = int(self.ptr.readline()[1:])
        self.seekbase = self.ptr.tell()
        self.ptr.seek(0, os.SEEK_END)
        self.n = (self.ptr.tell() - self.seekbase) // self.linelen
        self.lock = threading.Lock()

    def __len__(self):
        return self.n

    def read(self, n: int):
        """(n in the image file, image file, dict)."""
        if not 0 <= n < self.n:
            raise IndexError(f"record {n} of {self.n}")
        with self.lock:
            self.ptr.seek(self.seekbase + self.linelen * n)
            ln = self.ptr.readline().strip().split("\t")
        if len(ln) == 2:
            ln.append("")
        d = json.loads(ln[2], object_hook=_json_to_obj) if len(ln[2]) >= 2 else {}
        return int(ln[0]), ln[1], d

    def write(self, n: int, nextfile: int, extfile: str, jsondict=None):
        """Record n (-1 or >= len appends), as LSXFile.write."""
        if jsondict is None:
            out = "{}\t{}".format(nextfile, extfile)
        elif isinstance(jsondict, str):
            out = "{}\t{}\t{}".format(nextfile, extfile, jsondict)
        else:
            js = json.dumps(jsondict, indent=None, sort_keys=True, separators=(",", ":"),
                            default=_obj_to_json)
            out = "{}\t{}\t{}".format(nextfile, extfile, js)
        with self.lock:
            if len(out) + 1 > self.linelen:
                self._rewrite(len(out))
            line = "{{:<{}}}\n".format(self.linelen - 1).format(out)
            if n < 0 or n >= self.n:
                self.ptr.seek(0, os.SEEK_END)
                self.n += 1
            else:
                self.ptr.seek(self.seekbase + self.linelen * n)
            self.ptr.write(line)
            self.ptr.flush()

    def _rewrite(self, need: int):
        self.ptr.seek(self.seekbase)
        lines = [self.ptr.read(self.linelen).rstrip() for _ in range(self.n)]
        self.linelen = max([need] + [len(x) for x in lines]) + 1 + 4
        self.ptr.seek(0)
        self.ptr.truncate()
        self.ptr.write("#LSX\n{}\n# {}\n".format(self.filecomment, self.linelen))
        self.seekbase = self.ptr.tell()
        fmt = "{{:<{}}}\n".format(self.linelen - 1)
        for x in lines:
            self.ptr.write(fmt.format(x))

    def close(self):
        if self.ptr is not None:
            self.ptr.close()
            self.ptr = None


def load_lst_params(path: str, sel=None) -> list[dict]:
    """Per-record dicts {"src", "idx", ...the record's JSON keys} (the role of
    EMAN2's load_lst_params for initialize_data, programs/e2spa_make3d.py:223)."""
    lsx = LSXFile(path, True)
    base = os.path.dirname(os.path.abspath(path))
    out = []
    for i in (range(len(lsx)) if not sel else sel):
        n, f, d = lsx.read(i)
        # image paths are relative to the working directory (EMAN2 projects);
        # fall back to the list's own directory
        src = f if os.path.isabs(f) or os.path.exists(f) else os.path.join(base, f)
        rec = {"src": src, "idx": n}
        rec.update(d)
        out.append(rec)
    lsx.close()
    return out


def weights_from_scores(records: list[dict]) -> np.ndarray:
    """Particle weights from alignment scores as initialize_data forms them
    (programs/e2spa_make3d.py:248-292, without the keep-fraction exclusions):
    no scores -> 1; scores <= 0 (similarities) -> -score / max(-score)."""
    s = np.array([r.get("score", 2e5) for r in records], np.float64)
    if len(s) == 0:
        return s.astype(np.float32)
    if np.max(s) > 1e5:
        s = np.zeros(len(s)) - 1
    if np.all(s == 0):
        s = s + 1
    if np.min(s) < 0:
        s = -s
        s[s < 0] = 0
        s = s / np.max(s)
    return s.astype(np.float32)


def records_to_meta(records: list[dict], weights=None, apix: float = 1.0):
    """fr_particle metadata of LSX records: rotation and translation of
    xform.projection, weight, and the defocus / CTF constants of a "ctf"
    entry (EMAN2Ctf dict) when present."""
    from .particles import particle_meta
    n = len(records)
    rots = np.zeros((n, 3, 3), np.float32)
    shifts = np.zeros((n, 2), np.float32)
    defocus = np.zeros(n, np.float32)
    common = None
    for i, r in enumerate(records):
        xf = r.get("xform.projection", Transform())
        rots[i] = xf.rotation_block()
        shifts[i] = xf.get_trans_2d()
        c = r.get("ctf")
        if isinstance(c, dict) and "defocus" in c:
            defocus[i] = float(c["defocus"]) + float(r.get("defocus", 0.0))
            common = common or {k: float(c[k]) for k in ("voltage", "cs", "ampcont", "apix",
                                                         "dfdiff", "dfang") if k in c}
    w = weights_from_scores(records) if weights is None else np.asarray(weights, np.float32)
    return particle_meta(rots, shifts, w, ctf=common, defocus=defocus,
                         apix=(common or {}).get("apix", apix))


# ------------------------------------------------------------------ streaming

class StackStream:
    """Chunks of consecutive particles of one .mrcs stack, moved to HBM while
    the caller works on earlier ones.

    A reader thread fills one of two pinned host buffers with a chunk's raw
    bytes (readinto: page cache -> pinned memory, one copy); the consumer
    copies it to the device and widens it to float32 (fr_decode_images), both
    on a copy stream of their own, and yields the device images once torch's
    current stream has been ordered after them.  A pinned buffer is refilled
    only after its copy to the device has completed; the yielded images are
    marked in use on the current stream, so their memory is not reused for a
    later chunk before the work queued there (the insertion) is done."""

    def __init__(self, path: str, chunk: int = 2048, first: int = 0, count: int | None = None,
                 device=None, threads: int | None = None):
        import torch
        self.threads = threads or min(16, os.cpu_count() or 1)
        self.info = mrc_info(path)
        if not self.info.is_stack:
            raise ImageDimensionException(f"{path}: a particle stack (.mrcs) is expected")
        self.path, self.chunk, self.first = path, int(chunk), int(first)
        self.count = self.info.nimg - first if count is None else int(count)
        self.device = torch.device("cuda") if device is None else torch.device(device)
        nb = self.chunk * self.info.image_bytes
        self.pinned = [torch.empty(nb, dtype=torch.uint8, pin_memory=True) for _ in range(2)]
        self.raw = torch.empty(nb, dtype=torch.uint8, device=self.device)
        self.copy_stream = torch.cuda.Stream(device=self.device)
        self.bytes_read = 0

    def __len__(self):
        return (self.count + self.chunk - 1) // self.chunk

    def _fill(self, k, slot, copied, ready, fd, pool):
        n = min(self.chunk, self.count - k * self.chunk)
        if copied[slot] is not None:
            copied[slot].synchronize()          # its previous chunk is on the device
        mv = memoryview(self.pinned[slot].numpy())[: n * self.info.image_bytes]
        base = self.info.data_offset + (self.first + k * self.chunk) * self.info.image_bytes
        # page cache -> pinned memory by several threads (preadv drops the GIL)
        seg = max(1 << 20, -(-len(mv) // self.threads))

        def part(a):
            b = min(len(mv), a + seg)
            while a < b:
                r = os.preadv(fd, [mv[a:b]], base + a)
                if r <= 0:
                    raise ImageDimensionException(f"{self.path}: short read")
                a += r

        for fut in [pool.submit(part, a) for a in range(0, len(mv), seg)]:
            fut.result()
        self.bytes_read += len(mv)
        ready[k].set()

    def __iter__(self):
        import torch
        lib = _lib.load()
        nchunks = len(self)
        ready = [threading.Event() for _ in range(nchunks)]
        copied = [None, None]
        errors = []
        go = [threading.Semaphore(0) for _ in range(2)]

        def reader():
            from concurrent.futures import ThreadPoolExecutor
            try:
                fd = os.open(self.path, os.O_RDONLY)
                try:
                    with ThreadPoolExecutor(self.threads) as pool:
                        for k in range(nchunks):
                            if k >= 2:
                                go[k % 2].acquire()  # the consumer has issued chunk k-2's copy
                            self._fill(k, k % 2, copied, ready, fd, pool)
                finally:
                    os.close(fd)
            except Exception as e:                  # surfaced on the consumer side
                errors.append(e)
                for ev in ready:
                    ev.set()

        t = threading.Thread(target=reader, daemon=True)
        t.start()
        vals = self.info.image_values
        cs = self.copy_stream
        try:
            for k in range(nchunks):
                ready[k].wait()
                if errors:
                    raise errors[0]
                slot = k % 2
                n = min(self.chunk, self.count - k * self.chunk)
                nbytes = n * self.info.image_bytes
                cur = torch.cuda.current_stream(self.device)
                with torch.cuda.stream(cs):
                    self.raw[:nbytes].copy_(self.pinned[slot][:nbytes], non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(cs)
                    out = torch.empty((n, self.info.ny, self.info.nx), dtype=torch.float32,
                                      device=self.device)
                copied[slot] = ev
                if k + 2 < nchunks:
                    go[slot].release()
                _lib.check(lib.fr_decode_images(ctypes.c_void_p(self.raw.data_ptr()),
                                                self.info.mode, int(self.info.swap), n * vals,
                                                ctypes.c_void_p(out.data_ptr()),
                                                ctypes.c_void_p(cs.cuda_stream)))
                cur.wait_stream(cs)
                out.record_stream(cur)
                yield self.first + k * self.chunk, out
        finally:
            for g in go:
                g.release()
                g.release()
            t.join()


def insert_stack(recon, path: str, meta, chunk: int = 2048) -> int:
    """Streams a .mrcs stack into a set-up FourierReconstructor: chunk k+1 is
    read and copied while chunk k is inserted.  meta: fr_particle array for
    every image of the stack.  Returns the particles inserted."""
    sz = ctypes.sizeof(_lib.fr_particle)
    done = 0
    for first, imgs in StackStream(path, chunk):
        n = imgs.shape[0]
        m = (_lib.fr_particle * n).from_address(ctypes.addressof(meta) + first * sz)
        recon.insert_particles(imgs, m)
        done += n
    return done


def reconstruct_lst(recon, path: str, chunk: int = 2048, weights=None) -> int:
    """e2spa_make3d's reconstruction loop over an #LSX particle list
    (programs/e2spa_make3d.py:215-345): the records give each particle's
    image (file and index), xform.projection, CTF and score; weights follow
    initialize_data's score rule unless given; runs of consecutive images of
    one .mrcs stack are streamed from disk and inserted in list order into
    the set-up reconstructor `recon`.  Particles with weight <= 0 are skipped
    (:303-305).  Returns the number of particles read."""
    recs = load_lst_params(path)
    if not recs:
        return 0
    meta = records_to_meta(recs, weights)
    sz = ctypes.sizeof(_lib.fr_particle)
    runs = []                                   # (src, first index, first record, count)
    for i, r in enumerate(recs):
        if runs and runs[-1][0] == r["src"] and runs[-1][1] + runs[-1][3] == r["idx"]:
            src, first, start, count = runs[-1]
            runs[-1] = (src, first, start, count + 1)
        else:
            runs.append((r["src"], r["idx"], i, 1))
    done = 0
    for src, first, start, count in runs:
        for k0, imgs in StackStream(src, chunk, first=first, count=count):
            n = imgs.shape[0]
            m = (_lib.fr_particle * n).from_address(ctypes.addressof(meta) + (start + k0 - first) * sz)
            recon.insert_particles(imgs, m)
            done += n
    return done
