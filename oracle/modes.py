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


def slab_te10_field(mode, freq):
    """TE10-like mode of a guide loaded by a centred full-height slab (width w along
    the wide side u, permittivity eps_slab; eps_air outside): E = v Ev(x),
    Ev = cos(kd x) for |x| < w/2 and cos(kd w/2) sin(ka (a/2 - |x|)) / sin(ka (a - w)/2)
    outside (x measured from the centre of the wide side), beta from the dispersion
    relation (port2d.slab_beta).  Peak |Ev| = 1."""
    from .port2d import slab_beta
    o, uh, vh, nh = _frame(mode)
    a, w = mode["a"], mode["w"]
    k0 = 2 * np.pi * freq * np.sqrt(MU0 * EPS0)
    beta = slab_beta(a, w, mode["eps_slab"], freq, eps_air=mode["eps_air"])
    kd = np.sqrt(mode["eps_slab"] * k0 ** 2 - beta ** 2 + 0j)
    ka = np.sqrt(mode["eps_air"] * k0 ** 2 - beta ** 2 + 0j)
    outer = np.cos(kd * w / 2) / np.sin(ka * (a - w) / 2)

    def prof(x):
        ax = np.abs(x)
        return np.where(ax < w / 2, np.cos(kd * x), outer * np.sin(ka * (a / 2 - ax)))

    xs = np.linspace(-a / 2, a / 2, 4001)
    peak = np.abs(prof(xs)).max()

    def Et(X):
        X = np.atleast_2d(X)
        x = (X - o) @ uh - a / 2
        return (prof(x) / peak)[:, None] * vh[None, :].astype(np.complex128)
    return Et, nh, beta


def mode_metrics(mode, freq, eps_c, mu_r):
    """gamma, Z, V, Pz and the field callables at one frequency."""
    if mode.get("kind") == "SLAB_TE10":
        return _slab_metrics(mode, freq, mu_r)
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


def _slab_metrics(mode, freq, mu_r):
    w_ = 2 * np.pi * freq
    Et, nh, beta = slab_te10_field(mode, freq)
    gamma = 1j * beta
    fac = gamma / (1j * w_ * mu_r * MU0)

    def Ht(X):
        return fac * np.cross(nh[None, :], Et(X))

    p0 = np.asarray(mode["vpath"][0], dtype=np.float64)
    p1 = np.asarray(mode["vpath"][1], dtype=np.float64)
    x, wq = roots_legendre(24)
    s = 0.5 * (x + 1)
    X = p0[None, :] + s[:, None] * (p1 - p0)[None, :]
    V = -np.sum(0.5 * wq * (Et(X) @ (p1 - p0)))
    # Pz over the rectangle, split at the slab faces so every piece is smooth
    o, uh, vh, _ = _frame(mode)
    a, b, w = mode["a"], mode["b"], mode["w"]
    xq, wx = roots_legendre(32)
    cuts = [0.0, (a - w) / 2, (a + w) / 2, a]
    Pz = 0.0
    for u0, u1 in zip(cuts[:-1], cuts[1:]):
        U, Vv = np.meshgrid(u0 + 0.5 * (u1 - u0) * (xq + 1), 0.5 * b * (xq + 1), indexing="ij")
        W = np.outer(0.5 * (u1 - u0) * wx, 0.5 * b * wx).ravel()
        Xr = o[None, :] + U.ravel()[:, None] * uh[None, :] + Vv.ravel()[:, None] * vh[None, :]
        Pz = Pz + 0.5 * np.sum(W * (np.cross(Et(Xr), np.conj(Ht(Xr))) @ nh))
    Z = 0.5 * V * np.conj(V) / np.conj(Pz)
    return {"gamma": gamma, "Z": Z, "V": V, "Pz": Pz, "Et": Et, "Ht": Ht}

