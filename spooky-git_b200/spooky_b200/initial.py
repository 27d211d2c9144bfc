"""Seeded initial conditions in the reference's spectral layout.

The reference parses white-noise / mean-field keys but does not implement
them (src/fields/initflow.cu:79-98), so the random fields of the benchmark
configurations are generated here.

random_solenoidal: a divergence-free Gaussian random vector field whose
shell spectrum is E(k) ~ k^4 exp(-2 (k/kpeak)^2) (|u_k| ~ k exp(-(k/kpeak)^2)),
phases from numpy's PCG64 seeded with `seed`, rescaled so that the mean of
u_x^2 + u_y^2 + u_z^2 over the grid is 3 rms^2 (rms per component).
"""
import numpy as np


def grid(p):
    """Reference real-space grid x_i = -L/2 + L i/N (src/fields/initflow.cu:29-33)."""
    x = -p.lx / 2 + p.lx * np.arange(p.nx) / p.nx
    y = -p.ly / 2 + p.ly * np.arange(p.ny) / p.ny
    z = -p.lz / 2 + p.lz * np.arange(p.nz) / p.nz
    return np.meshgrid(x, y, z, indexing="ij")


def kvectors(p):
    kx = 2 * np.pi / p.lx * np.fft.fftfreq(p.nx, 1.0 / p.nx)
    ky = 2 * np.pi / p.ly * np.fft.fftfreq(p.ny, 1.0 / p.ny)
    kz = 2 * np.pi / p.lz * np.arange(p.nz // 2 + 1)
    return np.meshgrid(kx, ky, kz, indexing="ij")


def to_spectral(fields):
    """Real fields [F][nx][ny][nz] -> spectral [F][nx][ny][nz/2+1] (unnormalised D2Z)."""
    return np.stack([np.fft.rfftn(f) for f in fields])


def random_solenoidal(p, seed, kpeak=4.0, rms=1.0):
    """Real-space solenoidal random field [3][nx][ny][nz] (see module doc)."""
    rng = np.random.default_rng(seed)
    KX, KY, KZ = kvectors(p)
    K2 = KX ** 2 + KY ** 2 + KZ ** 2
    K = np.sqrt(K2)
    amp = np.where(K > 0, K * np.exp(-(K / kpeak) ** 2), 0.0)
    U = np.stack([(rng.standard_normal(K.shape) + 1j * rng.standard_normal(K.shape)) * amp for _ in range(3)])
    kdot = KX * U[0] + KY * U[1] + KZ * U[2]
    ik2 = np.where(K2 > 0, 1.0 / np.where(K2 > 0, K2, 1.0), 0.0)
    U[0] -= KX * kdot * ik2
    U[1] -= KY * kdot * ik2
    U[2] -= KZ * kdot * ik2
    R = np.stack([np.fft.irfftn(c, s=(p.nx, p.ny, p.nz), axes=(0, 1, 2)) for c in U])
    R *= rms / np.sqrt(np.mean(R ** 2))
    return R


def mhd_random_state(p, seed_u=1, seed_b=2, b0=(0.0, 0.0, 0.1), kpeak=4.0):
    """u and B independent random solenoidal fields (rms 1 per component),
    plus a uniform B0 added to the k=0 mode of B; spectral layout."""
    u = random_solenoidal(p, seed_u, kpeak=kpeak)
    B = random_solenoidal(p, seed_b, kpeak=kpeak)
    for c in range(3):
        B[c] += b0[c]
    return to_spectral(np.concatenate([u, B]))


def masked_noise_state(p, U, rel=1e-3, seed=7):
    """U plus solenoidal random content on the modes the 2/3 rule removes
    (|k_d| > (2/3) k_d,max on any axis), with L2 norm rel * |U|: a state
    whose dealiased-out modes carry real content, so that the step cannot
    take the path that skips them.  Velocity and magnetic triples stay
    divergence-free; a theta field gets scalar noise."""
    rng = np.random.default_rng(seed)
    KX, KY, KZ = kvectors(p)
    kmx = 2 * np.pi / p.lx * (p.nx // 2 - 1)
    kmy = 2 * np.pi / p.ly * (p.ny // 2 - 1)
    kmz = 2 * np.pi / p.lz * (p.nz // 2 - 1)
    outside = (np.abs(KX) > 2.0 / 3.0 * kmx) | (np.abs(KY) > 2.0 / 3.0 * kmy) | (np.abs(KZ) > 2.0 / 3.0 * kmz)
    K2 = KX ** 2 + KY ** 2 + KZ ** 2
    ik2 = np.where(K2 > 0, 1.0 / np.where(K2 > 0, K2, 1.0), 0.0)
    F = U.shape[0]
    N = np.zeros_like(U)
    for f in range(F):
        c = (rng.standard_normal(KX.shape) + 1j * rng.standard_normal(KX.shape)) * outside
        # a real field's spectrum (Hermitian on the kz = 0 and Nyquist planes)
        N[f] = np.fft.rfftn(np.fft.irfftn(c, s=(p.nx, p.ny, p.nz), axes=(0, 1, 2)))
    for base in [b for b in (0, 3) if b + 3 <= F and not (p.heat_equation)]:
        kdot = KX * N[base] + KY * N[base + 1] + KZ * N[base + 2]
        N[base] -= KX * kdot * ik2
        N[base + 1] -= KY * kdot * ik2
        N[base + 2] -= KZ * kdot * ik2
    N *= rel * np.linalg.norm(U.ravel()) / np.linalg.norm(N.ravel())
    return U + N
