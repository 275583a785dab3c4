"""VTK output of vesicle surfaces in the layout of the reference's WriteVTK
(src/StokesVelocity.cc:773-993) through the library's C ABI, and a reader of the files it
writes.

Per rank one XML PolyData file <fname>_<rank as 6 digits>.vtp with raw appended blocks,
and from rank 0 the index <fname>.pvtp. Per vesicle the points are the (p1+1) x 2p1 grid of
order p1 (latitude-major) and the poles at x = -1 and x = +1; the polygons are 2p1 pairs of
pole triangles, then p1 x 2p1 quads. The optional field is the point data "value".
"""
import re

import numpy as np

from ._lib import check, lib
from .stokes_velocity import _ptr


def _rank_size(rank, n_ranks):
    """The communicator of the reference's call: explicit rank and size, else those of the
    torch.distributed process group when one is up, else a single rank. Giving only one
    of rank and n_ranks is an error (the other would be guessed, and a wrong guess writes
    the index from the wrong process or makes piece names collide)."""
    if (rank is None) != (n_ranks is None):
        raise ValueError("give both rank and n_ranks, or neither")
    if rank is not None:
        return int(rank), int(n_ranks)
    try:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return dist.get_rank(), dist.get_world_size()
    except ImportError:  # pragma: no cover
        pass
    return 0, 1


def WriteVTK(S, p0, p1, fname, period=0.0, v=None, rank=None, n_ranks=None):
    """WriteVTK(S, p0, p1, fname, period, v_ptr, comm): surfaces S (and the field v) of order
    p0, float64 numpy arrays or CUDA tensors of [n_ves][3][(p0+1) 2p0], taken to order p1
    (p0 when p1 <= 0, like the Surface overload's order = -1) on the GPU and written."""
    p0 = int(p0)
    p1 = p0 if p1 <= 0 else int(p1)
    sp, dev, n = _ptr(S)
    per = 3 * 2 * p0 * (p0 + 1)
    if n % per:
        raise ValueError("S is not a whole number of order-p0 vector fields")
    vp = None
    if v is not None:
        vp, vdev, vn = _ptr(v)
        if vn != n or vdev != dev:
            raise ValueError("v must match S in size and location")
    r, size = _rank_size(rank, n_ranks)
    check(lib().ves3d_vtk_write(sp, vp, n // per, p0, p1, str(fname).encode(), float(period), r, size, dev),
          "WriteVTK")


def write_grid(X1, Xp, p1, fname, V1=None, Vp=None, period=0.0, rank=None, n_ranks=None):
    """The writer alone on host arrays (no GPU): X1 (and V1) [n_ves][3][(p1+1) 2p1] grid values
    of order p1, Xp (and Vp) [n_ves][3][2] pole values (x = -1, then x = +1); rank and size
    as WriteVTK's."""
    rank, n_ranks = _rank_size(rank, n_ranks)
    X1 = np.ascontiguousarray(X1, dtype=np.float64)
    Xp = np.ascontiguousarray(Xp, dtype=np.float64)
    ng = 2 * p1 * (p1 + 1)
    if X1.size % (3 * ng) or Xp.size != X1.size // ng * 2:
        raise ValueError("X1 / Xp sizes do not match order p1")
    if (V1 is None) != (Vp is None):
        raise ValueError("V1 and Vp go together")
    v1 = vp = None
    if V1 is not None:
        V1 = np.ascontiguousarray(V1, dtype=np.float64)
        Vp = np.ascontiguousarray(Vp, dtype=np.float64)
        if V1.size != X1.size or Vp.size != Xp.size:
            raise ValueError("V1 / Vp must match X1 / Xp")
        v1, vp = V1.ctypes.data, Vp.ctypes.data
    check(lib().ves3d_vtk_write_grid(X1.ctypes.data, Xp.ctypes.data, v1, vp, X1.size // (3 * ng), int(p1),
                                     str(fname).encode(), float(period), int(rank), int(n_ranks)), "write_grid")


def read_vtp(path):
    """A PolyData file with raw appended blocks, as this module writes it:
    dict(points [N][3], value [N][k] or None, connectivity, offsets, header)."""
    raw = open(path, "rb").read()
    tag = b'<AppendedData encoding="raw">'
    at = raw.index(tag)
    base = raw.index(b"_", at + len(tag)) + 1
    header = raw[:at].decode()
    order = "<" if 'byte_order="LittleEndian"' in header else ">"
    types = {"Float64": "f8", "Int32": "i4"}
    out = dict(header=header, value=None)
    for m in re.finditer(r'<DataArray type="(\w+)"(?: NumberOfComponents="(\d+)")? Name="(\w+)" '
                         r'format="appended" offset="(\d+)" />', header):
        typ, comps, name, off = m.group(1), m.group(2), m.group(3), int(m.group(4))
        nbytes = int(np.frombuffer(raw, dtype=order + "i4", count=1, offset=base + off)[0])
        dt = np.dtype(order + types[typ])
        a = np.frombuffer(raw, dtype=dt, count=nbytes // dt.itemsize, offset=base + off + 4).copy()
        if comps:
            a = a.reshape(-1, int(comps))
        out[{"Position": "points"}.get(name, name)] = a
    return out


def read_pvtp(path):
    """The piece file names an index file lists."""
    return re.findall(r'<Piece Source="([^"]+)"/>', open(path).read())


def SHC2Pole(shc, p, pole, stream=None):
    """SphericalHarmonics::SHC2Pole on CUDA float64 tensors: shc [n_fun][p(p+2)] ->
    pole [n_fun][2] (x = -1, then x = +1)."""
    a, dev, n = _ptr(shc)
    b, bdev, m = _ptr(pole)
    nc = p * (p + 2)
    if not (dev and bdev) or n % nc or m != n // nc * 2:
        raise ValueError("expected CUDA float64 tensors [n_fun][p(p+2)] and [n_fun][2]")
    check(lib().ves3d_sht_pole(a, n // nc, int(p), b, stream), "SHC2Pole")


__all__ = ["WriteVTK", "write_grid", "read_vtp", "read_pvtp", "SHC2Pole"]
