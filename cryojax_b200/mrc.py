"""MRC2014 images, image stacks and volumes (read and write).

Replaces cryojax/io/_mrc.py, which goes through the ``mrcfile`` package
(absent here).  This module reads and writes the MRC2014 layout itself: a
1024-byte header of 4-byte words (nx, ny, nz, mode, nxstart..nzstart,
mx, my, mz, cell lengths and angles, axis map, dmin/dmax/dmean, ispg,
nsymbt, extra words with EXTTYP and NVERSION, origin, "MAP ", the machine
stamp, rms, nlabl and ten 80-character labels), then nsymbt bytes of
extended header, then the data with x fastest.  The array returned is
[z][y][x] ([y][x] for a single image), as mrcfile returns it.

Conventions kept from the reference:
  * ``read_array_from_mrc`` converts to float64 unless ``mmap`` (as
    cryojax/io/_mrc.py:36-100 does) and reports the grid spacing as
    cell length / sampling, which must agree across axes;
  * image stacks (``.mrcs``) are written with ispg = 0 and mz = 1, volumes
    (``.mrc``) with ispg = 1 and mz = nz, single images with nz = 1
    (mrcfile's set_image_stack / set_volume).
"""

from __future__ import annotations

import os
import pathlib
import struct

import numpy as np

# MRC2014 data modes this module reads (mode -> dtype); writing uses mode 2.
_MODES = {0: np.int8, 1: np.int16, 2: np.float32, 6: np.uint16, 12: np.float16}
_HEADER_BYTES = 1024


def _suffix(filename) -> str:
    """'.mrc' or '.mrcs': the first suffix of an MRC file name (anything else is an OSError)."""
    first = (pathlib.Path(filename).suffixes or [None])[0]
    if first not in (".mrc", ".mrcs"):
        raise OSError(f"{str(filename)!r} is not an MRC file name: expected a '.mrc' or '.mrcs' suffix")
    return first


def _require_suffix(filename, wanted: str, what: str, ndim: int, array) -> None:
    """Writers: `what` goes to a file named *`wanted` and must be an `ndim`-dimensional array."""
    if _suffix(filename) != wanted:
        raise OSError(f"an MRC {what} is written to a '{wanted}' file, not {str(filename)!r}")
    if np.ndim(array) != ndim:
        raise ValueError(f"an MRC {what} is a {ndim}-D array; got {np.ndim(array)}-D")


def read_mrc_header(filename) -> dict:
    """The header fields this module uses, as a dict (endianness from the machine stamp)."""
    with open(filename, "rb") as f:
        raw = f.read(_HEADER_BYTES)
    if len(raw) < _HEADER_BYTES:
        raise ValueError(f"{filename}: shorter than an MRC header")
    stamp = raw[212:214]
    endian = ">" if stamp == b"\x11\x11" else "<"
    words = struct.unpack(endian + "10i6f3i3f2i", raw[0:96])
    nx, ny, nz, mode, nxs, nys, nzs, mx, my, mz = words[:10]
    cella, cellb = words[10:13], words[13:16]
    dmin, dmax, dmean = words[19:22]
    ispg, nsymbt = words[22], words[23]
    (nversion,) = struct.unpack(endian + "i", raw[108:112])
    origin = struct.unpack(endian + "3f", raw[196:208])
    return dict(nx=nx, ny=ny, nz=nz, mode=mode, start=(nxs, nys, nzs), sampling=(mx, my, mz), cella=cella,
                cellb=cellb, axes=words[16:19], dmin=dmin, dmax=dmax, dmean=dmean, ispg=ispg, nsymbt=nsymbt,
                nversion=nversion, origin=origin, endian=endian)


def _kind(h) -> str:
    if h["nz"] == 1:
        return "image"
    if h["ispg"] == 0:
        return "image_stack"
    if h["ispg"] >= 401:
        return "volume_stack"
    return "volume"


def read_array_from_mrc(filename, *, loads_grid_spacing: bool = False, mmap: bool = False,
                        permissive: bool = False):
    """Read an MRC file into a NumPy array (float64 unless ``mmap``).

    cryojax/io/_mrc.py:36-100.  With ``loads_grid_spacing`` also return the
    pixel / voxel size (cell length over sampling; all axes must agree).
    """
    _suffix(filename)
    h = read_mrc_header(filename)
    if h["mode"] not in _MODES:
        raise ValueError(f"{filename}: unsupported MRC data mode {h['mode']}")
    dtype = np.dtype(_MODES[h["mode"]]).newbyteorder(h["endian"])
    shape = (h["nz"], h["ny"], h["nx"])
    offset = _HEADER_BYTES + h["nsymbt"]
    count = int(np.prod(shape))
    if os.path.getsize(filename) < offset + count * dtype.itemsize and not permissive:
        raise ValueError(f"{filename}: file is shorter than its header says")
    if mmap:
        data = np.memmap(filename, dtype=dtype, mode="r", offset=offset, shape=shape)
    else:
        with open(filename, "rb") as f:
            f.seek(offset)
            data = np.frombuffer(f.read(count * dtype.itemsize), dtype=dtype).reshape(shape)
    kind = _kind(h)
    if kind == "image":
        data = data[0]
    if not mmap:
        data = data.astype(np.float64)
    if not loads_grid_spacing:
        return data
    n_axes = 2 if kind in ("image", "image_stack") else 3
    spacing = np.asarray([h["cella"][i] / h["sampling"][i] if h["sampling"][i] else 0.0 for i in range(n_axes)])
    if np.any(spacing == 0.0):
        raise ValueError("the MRC voxel size must be set to read the grid spacing; found 0")
    if not np.all(spacing == spacing[0]):
        raise ValueError(f"the MRC voxel size must be the same in all dimensions; found {spacing}")
    return data, float(spacing[0])


def _header_stats(data):
    """(min, max, mean, rms) of a float32 array for the MRC header.

    torch's multithreaded CPU reductions over a zero-copy view: one pass for
    min / max and one for mean / variance.  They agree with np.mean and
    np.std(dtype=float64) to well within the float32 the header stores, and
    take a sixth of the time of NumPy's float64 passes over a 420 MB stack.
    """
    import warnings

    import torch

    if data.size == 0:
        return 0.0, 0.0, 0.0, 0.0
    with warnings.catch_warnings():  # a read-only array is only read here
        warnings.simplefilter("ignore")
        t = torch.from_numpy(data).reshape(-1)
    lo, hi = torch.aminmax(t)
    var, mean = torch.var_mean(t, correction=0)
    return float(lo), float(hi), float(mean), float(var.sqrt())


def _write(array, spacing, filename, kind, overwrite):
    if os.path.exists(filename) and not overwrite:
        raise FileExistsError(f"{filename} exists; pass overwrite=True to replace it")
    data = np.ascontiguousarray(np.asarray(array, dtype=np.float32))
    if kind == "image":
        ny, nx = data.shape
        nz = 1
        mx, my, mz = nx, ny, 1
        ispg = 0
    else:
        nz, ny, nx = data.shape
        mx, my = nx, ny
        mz, ispg = (1, 0) if kind == "image_stack" else (nz, 1)
    d = float(np.asarray(spacing))
    dmin, dmax, dmean, rms = _header_stats(data)
    header = bytearray(_HEADER_BYTES)
    struct.pack_into("<10i", header, 0, nx, ny, nz, 2, 0, 0, 0, mx, my, mz)
    struct.pack_into("<6f", header, 40, d * mx, d * my, d * mz, 90.0, 90.0, 90.0)
    struct.pack_into("<3i", header, 64, 1, 2, 3)
    struct.pack_into("<3f", header, 76, dmin, dmax, dmean)
    struct.pack_into("<2i", header, 88, ispg, 0)
    struct.pack_into("<i", header, 108, 20141)
    struct.pack_into("<3f", header, 196, 0.0, 0.0, 0.0)
    header[208:212] = b"MAP "
    header[212:216] = b"\x44\x44\x00\x00"
    struct.pack_into("<f", header, 216, rms)
    struct.pack_into("<i", header, 220, 1)
    label = b"Created by cryojax_b200"
    header[224:224 + len(label)] = label
    header[224 + len(label):224 + 80] = b" " * (80 - len(label))
    if data.dtype.byteorder == ">":
        data = data.astype("<f4")
    with open(filename, "wb") as f:
        f.write(bytes(header))
        f.write(memoryview(data).cast("B"))


def _no_compression(compression):
    if compression is not None:
        raise NotImplementedError("compressed MRC files are not supported")


def write_image_to_mrc(image, pixel_size, filename, overwrite: bool = False, compression=None):
    """cryojax/io/_mrc.py:103-134 (suffix .mrc, a 2-D array)."""
    _no_compression(compression)
    _require_suffix(filename, ".mrc", "image", 2, image)
    _write(image, pixel_size, filename, "image", overwrite)


def write_image_stack_to_mrc(image_stack, pixel_size, filename, overwrite: bool = False, compression=None):
    """cryojax/io/_mrc.py:137-172 (suffix .mrcs, a 3-D array; written as an image stack)."""
    _no_compression(compression)
    _require_suffix(filename, ".mrcs", "image stack", 3, image_stack)
    _write(image_stack, pixel_size, filename, "image_stack", overwrite)


def write_volume_to_mrc(voxel_grid, voxel_size, filename, overwrite: bool = False, compression=None):
    """cryojax/io/_mrc.py:175-210 (suffix .mrc, a 3-D array; written as a volume)."""
    _no_compression(compression)
    _require_suffix(filename, ".mrc", "volume", 3, voxel_grid)
    _write(voxel_grid, voxel_size, filename, "volume", overwrite)
