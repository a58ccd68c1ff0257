"""Material models (oracle).

Constants and formulas follow src/OpenParEM3D/OpenParEM3D.cpp:216,373 and
src/OpenParEMCommon/OpenParEMmaterials.cpp:600-883.
"""
import numpy as np

EPS0 = 8.8541878176e-12          # src/OpenParEM3D/OpenParEM3D.cpp:216
MU0 = 4e-7 * np.pi


def k0(freq):
    return 2 * np.pi * freq * np.sqrt(MU0 * EPS0)


def relative_eps(freq, eps_r, tand, sigma):
    """eps_c/eps0: loss tangent eps_r(1-j tand) (OpenParEMmaterials.cpp:672) and
    conductivity eps_r - j sigma/(w eps0) (:674)."""
    w = 2 * np.pi * freq
    return eps_r * (1 - 1j * tand) - 1j * sigma / (w * EPS0)


def surface_resistance(freq, sigma, mu_r=1.0, Rz=0.0):
    """Temperature::get_Rs, OpenParEMmaterials.cpp:860-874: sqrt(pi f mu/sigma)
    times the Dmitriev-Zdorov/Simonovich roughness factor on Rz."""
    Rs = np.sqrt(np.pi * freq * MU0 * mu_r / sigma)
    if Rz == 0:
        return Rs
    r = Rz / (2 * np.sqrt(3) * 2 * (1 + np.sqrt(2)))
    Aflat = 36 * r * r
    delta = np.sqrt(1 / (np.pi * freq * MU0 * mu_r * sigma))
    factor = 1 + 84 * (np.pi * r * r / Aflat) / (1 + delta / r + delta * delta / (2 * r * r))
    return Rs * factor
