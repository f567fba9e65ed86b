"""Seeded synthetic SU(3) gauge configurations in the reference field layout.

The reference has no public dataset: it gauge-fixes configurations read from
files.  Benchmarks and tests therefore use the synthetic inputs the project's
configurations name, generated on the host in FP64 from a ``numpy`` seed:

* Haar-random SU(3) matrices: QR of a 3x3 complex Gaussian, the phases of
  R's diagonal moved into Q (Mezzadri 2007), then divided by a cube root of
  the determinant so that det = 1.
* Smooth fields ``U_mu(x) = exp(i*eps*H_mu(x))``, H traceless Hermitian with
  N(0,1) entries (exponentiated through its eigen-decomposition on the host, by
  scaling and squaring of a Taylor series on a CUDA device).
* Gauge transforms ``U_mu(x) -> g(x) U_mu(x) g(x+mu)^dagger``.

Fields come out as float64 arrays in the GpuPattern layout
(lattice/access_pattern/GpuPattern.hxx:53-56), parity-split site order
(lattice/SiteCoord.hxx:104-129), 18 reals per link.
"""
from __future__ import annotations

import numpy as np


def volume(size) -> int:
    return int(np.prod(size))


def lexicographic_to_split(size) -> np.ndarray:
    """Parity-split index s of every lexicographic site l = ((t*Nx+x)*Ny+y)*Nz+z."""
    V = volume(size)
    l = np.arange(V, dtype=np.int64)
    c = np.unravel_index(l, tuple(size))
    par = (c[0] + c[1] + c[2] + c[3]) & 1
    return l // 2 + par * (V // 2)


def forward_neighbour_lex(size, mu) -> np.ndarray:
    """Lexicographic index of x + mu for every lexicographic x (periodic)."""
    V = volume(size)
    c = list(np.unravel_index(np.arange(V, dtype=np.int64), tuple(size)))
    c[mu] = (c[mu] + 1) % size[mu]
    return np.ravel_multi_index(tuple(c), tuple(size))


def haar_su3(n: int, rng: np.random.Generator) -> np.ndarray:
    z = (rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))) / np.sqrt(2.0)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r, axis1=1, axis2=2)
    q = q * (d / np.abs(d))[:, None, :]
    det = np.linalg.det(q)
    return q / (det ** (1.0 / 3.0))[:, None, None]


def traceless_hermitian(n: int, rng: np.random.Generator) -> np.ndarray:
    a = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
    h = 0.5 * (a + np.conj(np.swapaxes(a, 1, 2)))
    tr = np.trace(h, axis1=1, axis2=2).real / 3.0
    return h - tr[:, None, None] * np.eye(3)[None]


def expi_hermitian(h: np.ndarray, eps: float) -> np.ndarray:
    w, v = np.linalg.eigh(h)
    return np.einsum("nij,nj,nkj->nik", v, np.exp(1j * eps * w), np.conj(v))


def smooth_links(size, eps: float, rng: np.random.Generator, chunk: int = 1 << 18) -> np.ndarray:
    """links[mu, l] (lexicographic l) = exp(i*eps*H), complex128 [4, V, 3, 3]."""
    V = volume(size)
    out = np.empty((4, V, 3, 3), dtype=np.complex128)
    for mu in range(4):
        for a in range(0, V, chunk):
            b = min(V, a + chunk)
            out[mu, a:b] = expi_hermitian(traceless_hermitian(b - a, rng), eps)
    return out


def hot_links(size, rng: np.random.Generator) -> np.ndarray:
    V = volume(size)
    return haar_su3(4 * V, rng).reshape(4, V, 3, 3)


def gauge_transform(links: np.ndarray, size, g: np.ndarray) -> np.ndarray:
    """U_mu(x) -> g(x) U_mu(x) g(x+mu)^dagger; g[l] lexicographic."""
    out = np.empty_like(links)
    for mu in range(4):
        fw = forward_neighbour_lex(size, mu)
        out[mu] = np.einsum("nij,njk,nlk->nil", g, links[mu], np.conj(g[fw]))
    return out


def to_gpupattern(links: np.ndarray, size, dtype=np.float64) -> np.ndarray:
    """complex [4, V(lexicographic), 3, 3] -> GpuPattern real array of V*72 entries."""
    V = volume(size)
    split = lexicographic_to_split(size)
    arr = np.empty((4, 3, 3, 2, V), dtype=dtype)
    re = np.transpose(links.real, (0, 2, 3, 1))  # [mu, i, j, l]
    im = np.transpose(links.imag, (0, 2, 3, 1))
    arr[:, :, :, 0, :][..., split] = re
    arr[:, :, :, 1, :][..., split] = im
    return arr.reshape(-1)


def from_gpupattern(U: np.ndarray, size) -> np.ndarray:
    """GpuPattern real array -> complex [4, V(lexicographic), 3, 3]."""
    V = volume(size)
    a = U.reshape(4, 3, 3, 2, V).astype(np.float64)
    split = lexicographic_to_split(size)
    c = a[:, :, :, 0, :][..., split] + 1j * a[:, :, :, 1, :][..., split]
    return np.transpose(c, (0, 3, 1, 2))


def landau_functional(links: np.ndarray) -> float:
    """F = sum Re tr U / (Nc*Nd*V) of complex links [4, V, 3, 3]."""
    return float(np.trace(links, axis1=2, axis2=3).real.sum() / (12.0 * links.shape[1]))


def _expm_taylor(a, squarings: int = 8, order: int = 14):
    """exp(a) for a batch of 3x3 matrices: Taylor series of a / 2^squarings, then squarings."""
    import torch

    b = a / float(2 ** squarings)
    eye = torch.eye(3, dtype=a.dtype, device=a.device).expand_as(a)
    out = eye.clone()
    term = eye.clone()
    for k in range(1, order + 1):
        term = term @ b / k
        out = out + term
    for _ in range(squarings):
        out = out @ out
    return out


def _haar_from_gaussian_torch(z):
    """haar_su3 on a batch of complex Gaussian 3x3 matrices, elementwise on the device: modified
    Gram-Schmidt of the columns gives the Q of the QR decomposition whose R has a positive real
    diagonal -- the phase-fixed Q of haar_su3 -- then Q / det(Q)^(1/3) (principal cube root), without
    batched LAPACK calls, which are slow for millions of 3x3 matrices on a GPU."""
    import torch

    def dot(a, b):  # a^dagger b over the rows, per matrix
        return (a.conj() * b).sum(dim=1)

    cols = [z[:, :, j] for j in range(3)]
    q = []
    for j in range(3):
        v = cols[j]
        for k in range(j):
            v = v - dot(q[k], v)[:, None] * q[k]
        q.append(v / torch.sqrt((v.conj() * v).real.sum(dim=1))[:, None])
    Q = torch.stack(q, dim=2)
    det = (Q[:, 0, 0] * (Q[:, 1, 1] * Q[:, 2, 2] - Q[:, 1, 2] * Q[:, 2, 1])
           - Q[:, 0, 1] * (Q[:, 1, 0] * Q[:, 2, 2] - Q[:, 1, 2] * Q[:, 2, 0])
           + Q[:, 0, 2] * (Q[:, 1, 0] * Q[:, 2, 1] - Q[:, 1, 1] * Q[:, 2, 0]))
    return Q / (det ** (1.0 / 3.0))[:, None, None]


def _torch_linalg(size, eps: float, seed: int, transform: bool, device: str):
    """The same construction with the dense linear algebra on a CUDA device (torch).

    The random numbers are drawn with numpy from the same seed and in the same order as
    the host path, so both paths build the same field up to rounding (~1e-15).
    """
    import torch

    V = volume(size)
    rng = np.random.default_rng(seed)
    links = torch.empty((4, V, 3, 3), dtype=torch.complex128, device=device)
    chunk = 1 << 18
    for mu in range(4):
        for a in range(0, V, chunk):
            b = min(V, a + chunk)
            h = torch.from_numpy(traceless_hermitian(b - a, rng)).to(device)
            links[mu, a:b] = _expm_taylor(1j * eps * h)
    f0 = float(torch.diagonal(links, dim1=2, dim2=3).real.sum().item() / (12.0 * V))
    if transform:
        z = (rng.standard_normal((V, 3, 3)) + 1j * rng.standard_normal((V, 3, 3))) / np.sqrt(2.0)
        g = torch.empty((V, 3, 3), dtype=torch.complex128, device=device)
        for a in range(0, V, 1 << 20):
            b = min(V, a + (1 << 20))
            g[a:b] = _haar_from_gaussian_torch(torch.from_numpy(z[a:b]).to(device))
        for mu in range(4):
            fw = torch.from_numpy(forward_neighbour_lex(size, mu)).to(device)
            links[mu] = torch.einsum("nij,njk,nlk->nil", g, links[mu], g[fw].conj())
    return links, f0


def _to_gpupattern_torch(links, size, dtype):
    """to_gpupattern on the device: complex [4, V, 3, 3] tensor -> GpuPattern tensor of V*72 reals."""
    import torch

    V = volume(size)
    split = torch.from_numpy(lexicographic_to_split(size)).to(links.device)
    tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
    arr = torch.empty((4, 3, 3, 2, V), dtype=tdt, device=links.device)
    arr[:, :, :, 0, :][..., split] = links.real.permute(0, 2, 3, 1).to(tdt)
    arr[:, :, :, 1, :][..., split] = links.imag.permute(0, 2, 3, 1).to(tdt)
    return arr.reshape(-1)


def smooth_config(size, eps: float, seed: int, transform: bool = True, dtype=np.float64, device=None,
                  as_tensor: bool = False):
    """The "known fixed point" input: exp(i*eps*H) links under a seeded Haar gauge transform.

    Returns (field in GpuPattern layout, functional of the untransformed field).  With
    device="cuda" the eigen/QR work runs on the GPU (for large lattices); the returned field
    is a host numpy array, or with as_tensor=True a tensor left on that device (the layout
    conversion then runs there too, which matters at 48^4 where the complex links are 3 GB).
    """
    if device is not None:
        links, f0 = _torch_linalg(size, eps, seed, transform, device)
        if as_tensor:
            U = _to_gpupattern_torch(links, size, dtype)
            del links
            return U, f0
        return to_gpupattern(links.cpu().numpy(), size, dtype), f0
    rng = np.random.default_rng(seed)
    links = smooth_links(size, eps, rng)
    f0 = landau_functional(links)
    if transform:
        links = gauge_transform(links, size, haar_su3(volume(size), rng))
    return to_gpupattern(links, size, dtype), f0


def hot_config(size, seed: int, dtype=np.float64):
    """Haar-random links (the 8^4 plain-method configuration)."""
    return to_gpupattern(hot_links(size, np.random.default_rng(seed)), size, dtype)


def gpupattern_to_timeslices(U: np.ndarray, size) -> np.ndarray:
    """GpuPattern array -> GpuPatternTimeslice array (access_pattern/GpuPatternTimeslice.hxx:57-62):
    slice t at offset 72*Vs*t is the GpuPattern array of its {1, Nx, Ny, Nz} lattice, whose
    parity split is by x+y+z.  This is the layout a Coulomb context imports."""
    nt, nx, ny, nz = (int(v) for v in size)
    vs = nx * ny * nz
    v = nt * vs
    t, x, y, z = (a.reshape(-1) for a in np.meshgrid(np.arange(nt), np.arange(nx), np.arange(ny), np.arange(nz),
                                                     indexing="ij"))
    l = ((t * nx + x) * ny + y) * nz + z
    s_full = l // 2 + ((t + x + y + z) % 2) * (v // 2)
    ls = (x * ny + y) * nz + z
    s_slice = ls // 2 + ((x + y + z) % 2) * (vs // 2)
    src = np.asarray(U).reshape(72, v)
    out = np.empty((nt, 72, vs), dtype=src.dtype)
    out[t, :, s_slice] = src[:, s_full].T
    return out.reshape(-1)
