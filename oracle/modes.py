"""Analytic rectangular-waveguide port modes (oracle).

The reference obtains port modes from its 2D solver (src/OpenParEM3D/port.cpp:5081-5176,
load_modeMetrics :5302-5453).  For homogeneously filled rectangular ports the
TE_mn mode is known in closed form; this module supplies gamma, Et, Ht, the
voltage V = -int E.dl along the port's voltage path and the PV impedance
Z = 0.5 V V* / Pz* (src/OpenParEM2D/fem2D.cpp:1819).  Et is normalised so its
peak transverse amplitude coefficient is 1 (the reference scales modes to
max |Et| = 1, port.cpp:2291-2335).  Ht is the field of the wave travelling out
of the 3D domain along the outward normal, H_t = (gamma/(j w mu)) n x E_t.
"""
import numpy as np
from scipy.special import roots_legendre
from .materials import MU0, EPS0


def _frame(mode):
    o = np.asarray(mode["origin"], dtype=np.float64)
    u = np.asarray(mode["u"], dtype=np.float64)
    v = np.asarray(mode["v"], dtype=np.float64)
    n = np.asarray(mode["normal"], dtype=np.float64)
    return o, u / np.linalg.norm(u), v / np.linalg.norm(v), n / np.linalg.norm(n)


def te_field(mode):
    o, uh, vh, nh = _frame(mode)
    a, b, m, n = mode["a"], mode["b"], mode["m"], mode["n"]
    ku, kv = m * np.pi / a, n * np.pi / b
    amp = max(ku, kv)

    def Et(X):
        X = np.atleast_2d(X)
        uu = (X - o) @ uh
        vv = (X - o) @ vh
        Eu = -(kv / amp) * np.cos(ku * uu) * np.sin(kv * vv)
        Ev = (ku / amp) * np.sin(ku * uu) * np.cos(kv * vv)
        return (Eu[:, None] * uh[None, :] + Ev[:, None] * vh[None, :]).astype(np.complex128)
    return Et, nh


def mode_metrics(mode, freq, eps_c, mu_r):
    """gamma, Z, V, Pz and the field callables at one frequency."""
    assert mode.get("kind", "TE") == "TE"
    w = 2 * np.pi * freq
    k0 = w * np.sqrt(MU0 * EPS0)
    a, b, m, n = mode["a"], mode["b"], mode["m"], mode["n"]
    kc2 = (m * np.pi / a) ** 2 + (n * np.pi / b) ** 2
    gamma = np.sqrt(complex(kc2 - k0 ** 2 * eps_c * mu_r))
    mu = mu_r * MU0
    Et, nh = te_field(mode)
    fac = gamma / (1j * w * mu)

    def Ht(X):
        E = Et(X)
        return fac * np.cross(nh[None, :], E)

    # voltage: V = -int_path E . dl
    p0 = np.asarray(mode["vpath"][0], dtype=np.float64)
    p1 = np.asarray(mode["vpath"][1], dtype=np.float64)
    x, wq = roots_legendre(24)
    s = 0.5 * (x + 1)
    X = p0[None, :] + s[:, None] * (p1 - p0)[None, :]
    V = -np.sum(0.5 * wq * (Et(X) @ (p1 - p0)))
    # Pz = 1/2 int (E x H*) . n over the rectangle
    o, uh, vh, _ = _frame(mode)
    xu, wu = roots_legendre(24)
    U, Vv = np.meshgrid(0.5 * a * (xu + 1), 0.5 * b * (xu + 1), indexing="ij")
    W = np.outer(0.5 * a * wu, 0.5 * b * wu).ravel()
    Xr = o[None, :] + U.ravel()[:, None] * uh[None, :] + Vv.ravel()[:, None] * vh[None, :]
    E = Et(Xr)
    H = Ht(Xr)
    Pz = 0.5 * np.sum(W * (np.cross(E, np.conj(H)) @ nh))
    Z = 0.5 * V * np.conj(V) / np.conj(Pz)
    return {"gamma": gamma, "Z": Z, "V": V, "Pz": Pz, "Et": Et, "Ht": Ht}
