"""Coil preprocessing for the real-data path on the GPU: SVD coil compression
(coil_compression.py:6-46) and 3-D ESPIRiT receive sensitivities (espirit.py:9-239).

Both keep the reference's function names, arguments and conventions (including its quirks, noted
below), take NumPy or CUDA arrays and return CUDA tensors.  The volume-sized work runs on the
GPU: the coil covariance and the compression are GEMMs over all voxels, the ESPIRiT calibration
matrix is gathered on the device, its line FFTs run on libmotionest's FFT kernels, and the
per-voxel coil eigenproblems are one batched eigendecomposition per plane.  The small dense
factorisations (a C x C SVD, the calibration matrix's SVD) are the library routines the
reference calls too.
"""
import numpy as np
import torch

from . import _lib
from ._arrays import to_device
from ._lib import ptr


def coil_compression(mps, ksp=None, perc=0.95, reg=1e-6):
    """Compress coils to the principal components holding `perc` of the energy.

    As coil_compression.py:6-46: P = sum over voxels of (mps / (sum_c |mps_c|^2 + reg)) mps^H,
    U S = svd(P), keep n = argmax(cumsum(S) / sum(S) >= perc) components (the reference's count:
    the index of the first component that reaches `perc`, so one fewer than the components
    needed), A = U^H[:n], and return (A mps, A ksp or None), shaped [n, ...].  The C x C SVD runs
    on the host in the precision of the inputs, as NumPy runs it for the reference."""
    _lib.require_cuda()
    m = to_device(mps, torch.complex64)
    C = m.shape[0]
    img_shape = tuple(m.shape[1:])
    M = m.reshape(C, -1)
    norm = 1.0 / (torch.sum(M.real * M.real + M.imag * M.imag, dim=0) + reg)
    P = (M * norm) @ M.conj().T  # [C, C]: one GEMM over all voxels
    U, S, _ = np.linalg.svd(P.cpu().numpy())
    energy = np.cumsum(S) / np.sum(S)
    n = int(np.argmax(energy >= perc))
    A = torch.as_tensor(np.ascontiguousarray(U.conj().T[:n]), device=m.device)
    cc_mps = (A @ M).reshape((n,) + img_shape)
    cc_ksp = None
    if ksp is not None:
        k = to_device(ksp, torch.complex64)
        cc_ksp = (A @ k.reshape(C, -1)).reshape((n,) + img_shape)
    return cc_mps, cc_ksp


def _fft_lines(v, axis, inverse):
    """Unnormalised FFT (numpy's convention: the inverse divides by N) along one of the first
    three axes of a [X, Y, Z, ...] complex64 CUDA tensor, on libmotionest's line kernels (which
    are orthonormal): the trailing dimensions become a batch of [X, Y, Z] volumes."""
    shp = tuple(v.shape)
    X, Y, Z = shp[:3]
    R = int(np.prod(shp[3:])) if len(shp) > 3 else 1
    w = v.reshape(X, Y, Z, R).permute(3, 0, 1, 2).contiguous()
    out = torch.empty_like(w)
    vox = X * Y * Z
    _lib.call("me_fft_axis", ptr(w), vox, ptr(out), vox, R, X, Y, Z, _lib.MeLayout(Y * Z, Z, 1),
              axis, int(inverse), _lib.stream_ptr())
    n = shp[axis]
    out = out * (1.0 / np.sqrt(n) if inverse else np.sqrt(n))
    return out.permute(1, 2, 3, 0).reshape(shp)


def _centred_ifft(v, axes):
    """fftshift(ifft(ifftshift(v))) along `axes` (numpy normalisation)."""
    v = torch.fft.ifftshift(v, dim=axes)
    for a in axes:
        v = _fft_lines(v, a, inverse=True)
    return torch.fft.fftshift(v, dim=axes)


def hankel_calibration(calib, kernel_size):
    """The calibration matrix of espirit.py:9-44: rows k + K c (k the kernel offset i + kx j +
    kx ky l, Fortran order; c the coil), columns the block positions (x fastest, then y, z)."""
    x = calib
    if x.dim() == 3:
        x = x[..., None]
    kx, ky, kz = kernel_size
    NRx = x.shape[3]
    u = x.unfold(0, kx, 1).unfold(1, ky, 1).unfold(2, kz, 1)  # [bx, by, bz, c, i, j, l]
    u = u.permute(3, 6, 5, 4, 2, 1, 0)                         # [c, l, j, i, bz, by, bx]
    K = kx * ky * kz
    return u.reshape(K * NRx, -1)


def rx_espirit_3d(calib, imsize, kernel_size=None, eig_thresh=0.02, mask_thresh=0.99):
    """3-D ESPIRiT receive sensitivities [Nx, Ny, Nz, NRx] from calibration k-space
    [NKx, NKy, NKz, NRx], as espirit.py:46-239: calibration matrix, its left singular vectors
    above eig_thresh (a ratio to the largest if < 1, else a count), the kernels zero-padded to
    the image size and inverse-FFT'd (z first, then x and y per plane), the principal
    eigenvector of each voxel's NRx x NRx matrix where sqrt(largest eigenvalue) * prod(imsize) /
    sqrt(prod(kernel_size)) > mask_thresh (zero elsewhere), and the phase of coil 0 removed."""
    _lib.require_cuda()
    if kernel_size is None:
        kernel_size = (5, 5, 5)
    cal = to_device(calib, torch.complex64)
    NRx = cal.shape[3]
    Nx, Ny, Nz = imsize
    kx, ky, kz = kernel_size
    H = hankel_calibration(cal, kernel_size)
    U, S, _ = torch.linalg.svd(H, full_matrices=False)
    if eig_thresh < 1:
        keep = S > S[0] * eig_thresh if S.numel() and float(S[0]) > 0 else torch.zeros_like(S, dtype=torch.bool)
        U = U[:, keep]
    else:
        U = U[:, :int(round(eig_thresh))]
    ncomp = U.shape[1]
    sens = torch.zeros((Nx, Ny, Nz, NRx), dtype=torch.complex64, device=cal.device)
    if ncomp == 0:
        return sens
    # U[i + kx j + kx ky l + K c, comp] -> [i, j, l, c, comp]
    Ur = U.reshape(NRx, kz, ky, kx, ncomp).permute(3, 2, 1, 0, 4)
    pz0 = int(np.ceil((Nz - kz) / 2))
    Uz = torch.zeros((kx, ky, Nz, NRx, ncomp), dtype=torch.complex64, device=cal.device)
    Uz[:, :, pz0:pz0 + kz] = Ur
    Uz = _centred_ifft(Uz, (2,))
    px0 = int(np.ceil((Nx - kx) / 2))
    py0 = int(np.ceil((Ny - ky) / 2))
    norm_factor = float(np.prod(imsize)) / np.sqrt(float(np.prod(kernel_size)))
    for z in range(Nz):
        t = torch.zeros((Nx, Ny, 1, NRx, ncomp), dtype=torch.complex64, device=cal.device)
        t[px0:px0 + kx, py0:py0 + ky, 0] = Uz[:, :, z]
        t = _centred_ifft(t, (0, 1))[:, :, 0]
        Mv = t.reshape(-1, NRx, ncomp)
        Cv = Mv @ Mv.transpose(1, 2).conj()
        w, V = torch.linalg.eigh(Cv)
        vec = V[:, :, -1]
        mask = torch.sqrt(torch.clamp(w[:, -1], min=0)) * norm_factor > mask_thresh
        sl = torch.where(mask[:, None], vec, torch.zeros_like(vec))
        sens[:, :, z] = sl.reshape(Nx, Ny, NRx)
    ph = torch.angle(sens[..., 0:1])
    return sens * torch.exp(-1j * ph)
