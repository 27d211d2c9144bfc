"""Initial conditions shared by the tests (reference grids and seeded fields)."""
import numpy as np


def grid(p):
    """Reference real-space grid x_i = -L/2 + L i/N (src/fields/initflow.cu:29-33)."""
    x = -p.lx / 2 + p.lx * np.arange(p.nx) / p.nx
    y = -p.ly / 2 + p.ly * np.arange(p.ny) / p.ny
    z = -p.lz / 2 + p.lz * np.arange(p.nz) / p.nz
    return np.meshgrid(x, y, z, indexing="ij")


def to_spectral(fields):
    """Real fields [F][nx][ny][nz] -> reference spectral layout (unnormalised D2Z)."""
    return np.stack([np.fft.rfftn(f) for f in fields])


def kvectors(p):
    kx = 2 * np.pi / p.lx * np.fft.fftfreq(p.nx, 1.0 / p.nx)
    ky = 2 * np.pi / p.ly * np.fft.fftfreq(p.ny, 1.0 / p.ny)
    kz = 2 * np.pi / p.lz * np.arange(p.nz // 2 + 1)
    return np.meshgrid(kx, ky, kz, indexing="ij")


def random_solenoidal(p, seed, kpeak=4.0, rms=1.0):
    """Solenoidal Gaussian random vector field with shell spectrum
    E(k) ~ k^4 exp(-2 (k/kpeak)^2), rescaled to the given rms (per-component
    mean of u^2 = rms^2); phases from numpy's PCG64 seeded with `seed`."""
    rng = np.random.default_rng(seed)
    KX, KY, KZ = kvectors(p)
    K2 = KX ** 2 + KY ** 2 + KZ ** 2
    K = np.sqrt(K2)
    amp = np.where(K > 0, K ** 2 * np.exp(-(K / kpeak) ** 2) / np.maximum(K, 1e-30), 0.0)
    shape = K.shape
    comps = []
    for _ in range(3):
        comps.append((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * amp)
    U = np.stack(comps)
    # Leray projection to divergence-free
    kdot = KX * U[0] + KY * U[1] + KZ * U[2]
    ik2 = np.where(K2 > 0, 1.0 / np.where(K2 > 0, K2, 1.0), 0.0)
    U[0] -= KX * kdot * ik2
    U[1] -= KY * kdot * ik2
    U[2] -= KZ * kdot * ik2
    # real fields via irfftn enforces Hermitian symmetry; then rescale
    R = np.stack([np.fft.irfftn(c, s=(p.nx, p.ny, p.nz), axes=(0, 1, 2)) for c in U])
    R *= rms / np.sqrt(np.mean(R ** 2))
    return R
