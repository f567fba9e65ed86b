"""Configuration-file formats of the reference, restated in numpy.

TEST INFRASTRUCTURE ONLY: the tests compare the library's GPU file transcoder
(gf_file_read / gf_file_write) against these functions, and these functions
are pinned byte for byte against the reference's own readers and writers
(oracle/ref_io.cpp) where the reference tree is present.

Arrays ``U`` are in the reference's GpuPattern order (18 reals per link,
index s + V*(k + 18*mu), k = 6*row + 2*col + c, s the parity-split site),
float64 unless stated.

Formats and the reference lines they follow:
  PLAIN       StandardPattern.hxx:53-56 + LinkFile.hxx:83-167: link (l, mu) at
              (4*l + mu)*18, l = ((t*Nx + x)*Ny + y)*Nz + z, no header
  HEADERONLY  FileHeaderOnly.hxx:72-103: opaque header, then PLAIN
  VOGT        FileVogt.hxx:60-108: shorts ndim, nc, extents, sizeof(real)
  ILDG        apps/ildg.cpp:26-238: LIME, big-endian doubles,
              ((((t*Nz + z)*Ny + y)*Nx + x)*4 + mu_f)*18, mu = mu_f + 1 mod 4
  QCDSTAG     apps/qcdstag.cpp:17-67: native doubles,
              ((mu*Nt + t)*Nz + z)*Ny + y)*Nx + x)*18, mu as stored
"""
from __future__ import annotations

import struct

import numpy as np

PLAIN, HEADERONLY, VOGT, ILDG, QCDSTAG = range(5)


def gpu_site_index(size) -> np.ndarray:
    """s(t, x, y, z): parity-split index of every site, shape (Nt, Nx, Ny, Nz) (SiteCoord.hxx:104-175)."""
    nt, nx, ny, nz = size
    t, x, y, z = np.meshgrid(*(np.arange(n) for n in size), indexing="ij")
    l = ((t * nx + x) * ny + y) * nz + z
    v = nt * nx * ny * nz
    return (l // 2 + ((t + x + y + z) % 2) * (v // 2)).astype(np.int64)


def _links_tx(U: np.ndarray, size) -> np.ndarray:
    """GpuPattern array -> (Nt, Nx, Ny, Nz, mu, 18)."""
    v = int(np.prod(size))
    g = U.reshape(4, 18, v)
    s = gpu_site_index(size)
    return np.moveaxis(g[:, :, s], (0, 1), (4, 5))


def _links_to_gpu(L: np.ndarray, size, dtype) -> np.ndarray:
    v = int(np.prod(size))
    out = np.empty((4, 18, v), dtype=dtype)
    s = gpu_site_index(size)
    out[:, :, s] = np.moveaxis(L, (4, 5), (0, 1))
    return out.reshape(-1)


def gpu_to_timeslice(U: np.ndarray, size) -> np.ndarray:
    """GpuPattern array -> GpuPatternTimeslice array (access_pattern/GpuPatternTimeslice.hxx:57-62:
    slice t at offset t*72*Vs holds the GpuPattern array of the {1, Nx, Ny, Nz} lattice, whose
    parity is that of x+y+z)."""
    nt = size[0]
    ssize = (1,) + tuple(size[1:])
    vs = int(np.prod(ssize))
    L = _links_tx(np.asarray(U), size)  # (t, x, y, z, mu, k)
    return np.concatenate([_links_to_gpu(L[t:t + 1], ssize, np.asarray(U).dtype) for t in range(nt)]).reshape(
        nt * 72 * vs)


def timeslice_to_gpu(T: np.ndarray, size) -> np.ndarray:
    nt = size[0]
    ssize = (1,) + tuple(size[1:])
    vs = int(np.prod(ssize))
    T = np.asarray(T).reshape(nt, 72 * vs)
    L = np.concatenate([_links_tx(T[t], ssize) for t in range(nt)], axis=0)
    return _links_to_gpu(L, size, T.dtype)


def payload_encode(U: np.ndarray, size, fmt: int, file_dtype=np.float64) -> bytes:
    """The configuration payload (no header) of format fmt."""
    L = _links_tx(np.asarray(U), size)  # (t, x, y, z, mu, k)
    if fmt in (PLAIN, HEADERONLY, VOGT):
        return np.ascontiguousarray(L).astype(file_dtype).tobytes()
    if fmt == ILDG:
        Lf = np.roll(L, -1, axis=4)  # file mu_f holds internal mu = mu_f + 1
        Lf = np.transpose(Lf, (0, 3, 2, 1, 4, 5))  # t, z, y, x, mu_f, k
        return np.ascontiguousarray(Lf).astype(">f8").tobytes()
    if fmt == QCDSTAG:
        Lf = np.transpose(L, (4, 0, 3, 2, 1, 5))  # mu, t, z, y, x, k
        return np.ascontiguousarray(Lf).astype("<f8").tobytes()
    raise ValueError(fmt)


def payload_decode(data: bytes, size, fmt: int, file_dtype=np.float64, dtype=np.float64) -> np.ndarray:
    nt, nx, ny, nz = size
    if fmt in (PLAIN, HEADERONLY, VOGT):
        L = np.frombuffer(data, dtype=file_dtype).reshape(nt, nx, ny, nz, 4, 18)
    elif fmt == ILDG:
        Lf = np.frombuffer(data, dtype=">f8").reshape(nt, nz, ny, nx, 4, 18)
        L = np.roll(np.transpose(Lf, (0, 3, 2, 1, 4, 5)), 1, axis=4)
    elif fmt == QCDSTAG:
        Lf = np.frombuffer(data, dtype="<f8").reshape(4, nt, nz, ny, nx, 18)
        L = np.transpose(Lf, (1, 4, 3, 2, 0, 5))
    else:
        raise ValueError(fmt)
    return _links_to_gpu(L.astype(np.float64), size, dtype)


def vogt_header(size, real_bytes: int) -> bytes:
    return struct.pack("=7h", 4, 3, *size, real_bytes)


# ---- LIME (the SciDAC container the ILDG format uses) --------------------------------------------
LIME_MAGIC = 0x456789AB


def lime_record(rtype: str, data: bytes, mb: bool, me: bool) -> bytes:
    flags = (0x8000 if mb else 0) | (0x4000 if me else 0)
    head = struct.pack(">IHHQ", LIME_MAGIC, 1, flags, len(data)) + rtype.encode().ljust(128, b"\0")
    return head + data + b"\0" * ((-len(data)) % 8)


def lime_records(blob: bytes) -> list[tuple[str, bytes, bool, bool]]:
    out, pos = [], 0
    while pos < len(blob):
        magic, _ver, flags, n = struct.unpack(">IHHQ", blob[pos:pos + 16])
        if magic != LIME_MAGIC:
            raise ValueError("bad LIME magic")
        rtype = blob[pos + 16:pos + 144].split(b"\0", 1)[0].decode()
        data = blob[pos + 144:pos + 144 + n]
        out.append((rtype, data, bool(flags & 0x8000), bool(flags & 0x4000)))
        pos += 144 + n + ((-n) % 8)
    return out


def ildg_file(U: np.ndarray, size, extra: list[tuple[str, bytes]] = ()) -> bytes:
    """A LIME file: the records `extra` (type, text) in order, then ildg-binary-data."""
    recs = list(extra) + [("ildg-binary-data", payload_encode(U, size, ILDG))]
    return b"".join(lime_record(t, d, i == 0, i == len(recs) - 1) for i, (t, d) in enumerate(recs))


def ildg_rewrite(template: bytes, U: np.ndarray, size, sa_steps: int) -> bytes:
    """What writeILDG makes of a template file (apps/ildg.cpp:99-238): records copied in order,
    text records cut at their first NUL, " SA steps N" appended to xlf-info, new binary data."""
    out = []
    for rtype, data, mb, me in lime_records(template):
        if rtype == "ildg-binary-data":
            new = payload_encode(U, size, ILDG)
        else:
            text = data.split(b"\0", 1)[0]
            new = text + (b" SA steps %d" % sa_steps if rtype == "xlf-info" else b"")
        out.append(lime_record(rtype, new, mb, me))
    return b"".join(out)


def random_links(size, seed: int) -> np.ndarray:
    """Random reals in GpuPattern order (file transcoding does not care about unitarity)."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal(72 * int(np.prod(size)))
