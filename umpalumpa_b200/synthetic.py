"""Seeded synthetic Fourier-reconstruction inputs (bench and test data, not the product path).

A job is ``n`` projections of a phantom made of 40 isotropic 3D Gaussians (sigma U(2,6)
voxels, amplitude U(0.5,1), centres uniform in a ball of radius B/4 about the box centre),
each viewed under a Haar-uniform random rotation R (from a uniform unit quaternion), plus
white Gaussian noise with variance var(signal)/SNR.  The projection along R*z of a Gaussian
of amplitude a and width s is a 2D Gaussian of amplitude a*s*sqrt(2*pi) centred at the
projection of its centre on the image axes R*x, R*y; images are B x B, centred at B/2.

Each image is real-FFT'd into a half-plane of X = B/2+1 columns and Y = B rows and then
prepared the way the reference's Fourier-processing step prepares it for insertion
(libumpalumpa/operations/fourier_processing/fp_cpu_kernels.hpp:21-37, centre + normalise +
shift, no crop): rows are shifted so that DC sits at y = Y/2, every coefficient is scaled by
1/B^2 and by (-1)^(x+y) of its unshifted position.  The traverse-space transform of a
projection is R itself, so frequency (kx, ky) lands at R*(kx, ky, 0).

The ``numpy`` backend is used for parity cases; the ``torch`` backend builds production-size
jobs directly in device memory with the same recipe (the two do not share random streams).
"""
from __future__ import annotations

import math

import numpy as np

N_GAUSSIANS = 40


def quaternion_rotations(n: int, rng: np.random.Generator) -> np.ndarray:
    """n Haar-uniform rotations as float32 [n,3,3] (unit quaternion -> matrix)."""
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    m = np.empty((n, 3, 3), np.float64)
    m[:, 0, 0] = 1 - 2 * (y * y + z * z)
    m[:, 0, 1] = 2 * (x * y - z * w)
    m[:, 0, 2] = 2 * (x * z + y * w)
    m[:, 1, 0] = 2 * (x * y + z * w)
    m[:, 1, 1] = 1 - 2 * (x * x + z * z)
    m[:, 1, 2] = 2 * (y * z - x * w)
    m[:, 2, 0] = 2 * (x * z - y * w)
    m[:, 2, 1] = 2 * (y * z + x * w)
    m[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return m.astype(np.float32)


def phantom(box: int, rng: np.random.Generator):
    """Gaussian centres (relative to the box centre), widths and amplitudes."""
    d = rng.standard_normal((N_GAUSSIANS, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rad = (box / 4.0) * rng.random(N_GAUSSIANS) ** (1.0 / 3.0)
    centres = d * rad[:, None]
    sigma = rng.uniform(2.0, 6.0, N_GAUSSIANS)
    amp = rng.uniform(0.5, 1.0, N_GAUSSIANS)
    return centres, sigma, amp


def _prepare_halfplanes_np(img: np.ndarray) -> np.ndarray:
    n, b, _ = img.shape
    f = np.fft.rfft2(img.astype(np.float64), axes=(1, 2))  # [n, Y, X]
    yy = np.arange(b)[:, None]
    xx = np.arange(b // 2 + 1)[None, :]
    sign = 1.0 - 2.0 * ((xx + yy) & 1)
    f = f * (sign / float(b * b))
    return np.roll(f, b // 2, axis=1).astype(np.complex64)


def make_job(box: int, n: int, seed: int, snr: float = 0.1):
    """Return (halfplanes complex64 [n, B, B/2+1], rotations float32 [n,3,3]) via numpy."""
    rng = np.random.default_rng(seed)
    centres, sigma, amp = phantom(box, rng)
    rots = quaternion_rotations(n, rng)
    u = np.arange(box, dtype=np.float64) - box / 2.0
    out = np.empty((n, box, box // 2 + 1), np.complex64)
    chunk = 256
    for s in range(0, n, chunk):
        r = rots[s:s + chunk].astype(np.float64)
        cu = np.einsum("kj,njc->nkc", centres, r)  # centre . (R x), centre . (R y), centre . (R z)
        a = amp * sigma * math.sqrt(2 * math.pi)
        gu = np.exp(-((u[None, None, :] - cu[:, :, 0:1]) ** 2) / (2 * sigma[None, :, None] ** 2))
        gv = np.exp(-((u[None, None, :] - cu[:, :, 1:2]) ** 2) / (2 * sigma[None, :, None] ** 2))
        img = np.einsum("nkv,nku->nvu", gv * a[None, :, None], gu)
        var = img.reshape(len(r), -1).var(axis=1)
        noise = rng.standard_normal(img.shape) * np.sqrt(var / snr)[:, None, None]
        out[s:s + chunk] = _prepare_halfplanes_np(img + noise)
    return out, rots


def make_job_torch(box: int, n: int, seed: int, snr: float, device, out=None, chunk: int = 1024):
    """The same recipe in torch on `device`, writing half-planes into `out` (complex64
    [n, B, B/2+1], allocated when None).  Rotations are returned as float32 numpy [n,3,3]."""
    import torch

    rng = np.random.default_rng(seed)
    centres, sigma, amp = phantom(box, rng)
    rots = quaternion_rotations(n, rng)
    if out is None:
        out = torch.empty((n, box, box // 2 + 1), dtype=torch.complex64, device=device)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    u = torch.arange(box, dtype=torch.float32, device=device) - box / 2.0
    c = torch.as_tensor(centres, dtype=torch.float32, device=device)
    sg = torch.as_tensor(sigma, dtype=torch.float32, device=device)
    a = torch.as_tensor(amp * sigma * math.sqrt(2 * math.pi), dtype=torch.float32, device=device)
    yy = torch.arange(box, device=device)[:, None]
    xx = torch.arange(box // 2 + 1, device=device)[None, :]
    sign = (1.0 - 2.0 * ((xx + yy) & 1).float()) / float(box * box)
    for s in range(0, n, chunk):
        r = torch.as_tensor(rots[s:s + chunk], dtype=torch.float32, device=device)
        cu = torch.einsum("kj,njc->nkc", c, r)
        gu = torch.exp(-((u[None, None, :] - cu[:, :, 0:1]) ** 2) / (2 * sg[None, :, None] ** 2))
        gv = torch.exp(-((u[None, None, :] - cu[:, :, 1:2]) ** 2) / (2 * sg[None, :, None] ** 2))
        img = torch.einsum("nkv,nku->nvu", gv * a[None, :, None], gu)
        var = img.reshape(len(r), -1).var(dim=1)
        img = img + torch.randn(img.shape, generator=g, device=device) * torch.sqrt(var / snr)[:, None, None]
        f = torch.fft.rfft2(img) * sign
        out[s:s + chunk] = torch.roll(f, box // 2, dims=1).to(torch.complex64)
    return out, rots


SERVED_BOXES = (64, 96, 128, 192, 256, 320)


def served_trace(n_jobs: int, seed: int = 0, rate: float = 20.0, boxes=SERVED_BOXES,
                 total_range=(2000, 30000), batch_range=(256, 4096), gap_mean: float = 0.010):
    """Arrival trace of the served workload: jobs arrive by a Poisson process (`rate` jobs/s),
    each with a box drawn uniformly from `boxes` and a projection count uniform over
    `total_range`, streamed as batches of uniform size over `batch_range` whose arrivals are
    separated by exponential gaps of mean `gap_mean` seconds, the first at the job's arrival.

    Returns a list of dicts {job, arrival, box, total, batches: [(time, n), ...]} sorted by
    arrival; every draw comes from one generator seeded with `seed`."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for j in range(n_jobs):
        t += float(rng.exponential(1.0 / rate))
        box = int(boxes[int(rng.integers(len(boxes)))])
        total = int(rng.integers(total_range[0], total_range[1] + 1))
        batches, left, bt = [], total, t
        while left > 0:
            n = min(left, int(rng.integers(batch_range[0], batch_range[1] + 1)))
            batches.append((bt, n))
            left -= n
            bt += float(rng.exponential(gap_mean))
        jobs.append({"job": j, "arrival": t, "box": box, "total": total, "batches": batches})
    return jobs
