// S-parameter post-processing on the host: renormalisation to a reference
// impedance, mixed-mode conversion, Touchstone 1.1 / 2.0 and results-CSV output,
// and the regression comparator (test cases against a results CSV) (the reference's Result::S2Z / Z2S /
// renormalize, src/OpenParEM3D/results.cpp:455-580, and
// ResultDatabase::saveTouchstone, results.cpp:1055-1208).  The file layout
// follows the Touchstone 1.1 conventions the reference writes: "# <unit> S
// <RI|MA|DB> R <Zref>", 1- and 2-port data with S11 S21 S12 S22 (column by
// column) on one line per frequency, more ports row by row with at most four
// pairs per line and a "!row i" comment, 15 significant digits.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/opem_b200.h"

namespace {

using cd = std::complex<double>;

// inverse of an n x n complex matrix (row-major) by Gauss-Jordan with partial
// pivoting; false when a pivot is not above rel_tol times the largest entry
bool invert(int n, std::vector<cd>& a, double rel_tol = 0.0) {
    double amax = 0.0;
    for (const cd& v : a) amax = std::max(amax, std::abs(v));
    const double tiny = rel_tol * amax;
    std::vector<cd> inv((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r)
            if (std::abs(a[(size_t)r * n + c]) > std::abs(a[(size_t)p * n + c])) p = r;
        if (!(std::abs(a[(size_t)p * n + c]) > tiny)) return false;
        if (p != c)
            for (int k = 0; k < n; ++k) {
                std::swap(a[(size_t)p * n + k], a[(size_t)c * n + k]);
                std::swap(inv[(size_t)p * n + k], inv[(size_t)c * n + k]);
            }
        const cd d = 1.0 / a[(size_t)c * n + c];
        for (int k = 0; k < n; ++k) {
            a[(size_t)c * n + k] *= d;
            inv[(size_t)c * n + k] *= d;
        }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const cd f = a[(size_t)r * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) {
                a[(size_t)r * n + k] -= f * a[(size_t)c * n + k];
                inv[(size_t)r * n + k] -= f * inv[(size_t)c * n + k];
            }
        }
    }
    a.swap(inv);
    return true;
}

std::vector<cd> matmul(int n, const std::vector<cd>& a, const std::vector<cd>& b) {
    std::vector<cd> c((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j) c[(size_t)i * n + j] += a[(size_t)i * n + k] * b[(size_t)k * n + j];
    return c;
}

// Writes one frequency point's S in the reference's data layout (shared by the
// Touchstone 1.1 and 2.0 writers).
void write_point(FILE* f, int n, const double* Sq, double fscaled, const std::string& fmt) {
    auto pair = [&](const cd& v) {
        double a, b;
        if (fmt == "RI") { a = v.real(); b = v.imag(); }
        else if (fmt == "MA") { a = std::abs(v); b = std::arg(v) * 180.0 / M_PI; }
        else { a = 20.0 * std::log10(std::abs(v)); b = std::arg(v) * 180.0 / M_PI; }
        std::fprintf(f, " %.15g %.15g", a, b);
    };
    auto at = [&](int r, int c) { return cd(Sq[2 * (r * n + c)], Sq[2 * (r * n + c) + 1]); };
    std::fprintf(f, "%.15g", fscaled);
    if (n < 3) {
        for (int col = 0; col < n; ++col)
            for (int row = 0; row < n; ++row) pair(at(row, col));
        std::fprintf(f, "\n");
    } else {
        for (int row = 0; row < n; ++row)
            for (int col = 0; col < n; ++col) {
                pair(at(row, col));
                const int cnt = col + 1;
                if (cnt % 4 == 0 || cnt == n) {
                    if (cnt <= 4) std::fprintf(f, " !row %d", row + 1);
                    std::fprintf(f, "\n");
                }
            }
    }
}

double unit_scale(const std::string& un) {
    if (un == "Hz") return 1;
    if (un == "kHz") return 1e-3;
    if (un == "MHz") return 1e-6;
    if (un == "GHz") return 1e-9;
    return 0;
}

}  // namespace

extern "C" {

// Mixed-mode conversion, fem3D::build_Mc_Ms with conversion = 1
// (src/OpenParEM3D/fem3D.cpp:1586-1900) and Result::SparameterConversion
// (results.cpp:587-630, Meyer and Prinsloo, IEEE TAP 63(11) 2015, eq. 15):
// for each pair (P, N) the common mode takes S-port P with Zoe = zref/2 and the
// differential mode S-port N with Zoo = 2 zref; Kv maps (Vp, Vn) to
// ((Vp+Vn)/2, Vp-Vn) and Ki maps (Ip, In) to (Ip+In, (Ip-In)/2), identity elsewhere;
// term1 = Zb^-1/2 Kv Za^1/2, term2 = Zb^1/2 Ki Za^-1/2, Ms = (term1+term2)/2,
// Mc = (term1-term2)/2, S_b = (Mc + Ms S)(Ms + Mc S)^-1.
int opem_s_mixed_mode(int nports, const double* S, int npairs, const int* pairs, double zref, double* S_out,
                      double* Zo_out) {
    if (nports < 1 || !S || npairs < 0 || (npairs > 0 && !pairs) || !(zref > 0) || !S_out) return OPEM_ERR_ARG;
    const int n = nports;
    std::vector<int> used(n, 0);
    for (int k = 0; k < npairs; ++k) {
        const int p = pairs[2 * k] - 1, q = pairs[2 * k + 1] - 1;
        if (p < 0 || p >= n || q < 0 || q >= n || p == q || used[p] || used[q]) return OPEM_ERR_ARG;
        used[p] = used[q] = 1;
    }
    const double Zoe = zref / 2, Zoo = zref * 2;
    std::vector<double> za(n, zref), zb(n, zref);
    for (int k = 0; k < npairs; ++k) {
        zb[pairs[2 * k] - 1] = Zoe;
        zb[pairs[2 * k + 1] - 1] = Zoo;
    }
    std::vector<cd> Kv((size_t)n * n, 0.0), Ki((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) Kv[(size_t)i * n + i] = Ki[(size_t)i * n + i] = 1.0;
    for (int k = 0; k < npairs; ++k) {
        const int p = pairs[2 * k] - 1, q = pairs[2 * k + 1] - 1;
        Kv[(size_t)p * n + p] = 0.5; Kv[(size_t)p * n + q] = 0.5;
        Kv[(size_t)q * n + p] = 1.0; Kv[(size_t)q * n + q] = -1.0;
        Ki[(size_t)p * n + p] = 1.0; Ki[(size_t)p * n + q] = 1.0;
        Ki[(size_t)q * n + p] = 0.5; Ki[(size_t)q * n + q] = -0.5;
    }
    std::vector<cd> Ms((size_t)n * n), Mc((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const cd t1 = Kv[(size_t)i * n + j] * std::sqrt(za[j]) / std::sqrt(zb[i]);
            const cd t2 = Ki[(size_t)i * n + j] * std::sqrt(zb[i]) / std::sqrt(za[j]);
            Ms[(size_t)i * n + j] = 0.5 * (t1 + t2);
            Mc[(size_t)i * n + j] = 0.5 * (t1 - t2);
        }
    std::vector<cd> Sa((size_t)n * n);
    for (int i = 0; i < n * n; ++i) Sa[i] = cd(S[2 * i], S[2 * i + 1]);
    std::vector<cd> num = matmul(n, Ms, Sa), den = matmul(n, Mc, Sa);
    for (int i = 0; i < n * n; ++i) { num[i] += Mc[i]; den[i] += Ms[i]; }
    if (!invert(n, den)) return OPEM_ERR_BREAKDOWN;
    std::vector<cd> Sb = matmul(n, num, den);
    for (int i = 0; i < n * n; ++i) { S_out[2 * i] = Sb[i].real(); S_out[2 * i + 1] = Sb[i].imag(); }
    if (Zo_out)
        for (int i = 0; i < n; ++i) { Zo_out[2 * i] = zb[i]; Zo_out[2 * i + 1] = 0.0; }
    return OPEM_OK;
}

// Line-to-modal maps of a port with n conductors carrying n modes, the
// reference's "line" calculation (OpenParEM2D Mode::calculateModalCurrent /
// calculateModalVoltage, src/OpenParEM2D/fem2D.cpp:1591-1790): for mode i with
// currents I[i][k] on the lines' current paths, Ti[i][k] = sign(Re I[i][k]) times
// 0.5 (|sum_k sign I| + |sum_k I|) / |sum_k sign I| (the return current); a mode
// whose Ti[i][0] comes out negative has its field, currents and voltages flipped
// and its row negated; the mode current is sum_k Ti[i][k] I[i][k]; then
// Tv = (conj(Ti)^-1)^T and the mode voltage sum_k Tv[i][k] V[i][k].
int opem_port_line_maps(int n, const double* I, const double* V, double* Ti, double* Tv, int* flipped, double* Im,
                        double* Vm) {
    if (n < 1 || !I || !Ti || !Tv) return OPEM_ERR_ARG;
    std::vector<cd> cur((size_t)n * n), vol((size_t)n * n, 0.0), T((size_t)n * n), K((size_t)n * n);
    for (int i = 0; i < n * n; ++i) {
        cur[i] = cd(I[2 * i], I[2 * i + 1]);
        if (V) vol[i] = cd(V[2 * i], V[2 * i + 1]);
    }
    std::vector<cd> mcur(n), mvol(n, 0.0);
    for (int i = 0; i < n; ++i) {
        cd mode_current = 0.0, return_current = 0.0;
        for (int k = 0; k < n; ++k) {
            const double sg = cur[(size_t)i * n + k].real() >= 0 ? 1.0 : -1.0;
            T[(size_t)i * n + k] = sg;
            mode_current += sg * cur[(size_t)i * n + k];
            return_current += cur[(size_t)i * n + k];
        }
        if (!(std::abs(mode_current) > 0)) return OPEM_ERR_BREAKDOWN;
        const double scale = 0.5 * (std::abs(mode_current) + std::abs(return_current)) / std::abs(mode_current);
        for (int k = 0; k < n; ++k) T[(size_t)i * n + k] *= scale;
        int fl = 0;
        if (T[(size_t)i * n].real() < 0) {
            fl = 1;
            for (int k = 0; k < n; ++k) {
                T[(size_t)i * n + k] = -T[(size_t)i * n + k];
                cur[(size_t)i * n + k] = -cur[(size_t)i * n + k];
                vol[(size_t)i * n + k] = -vol[(size_t)i * n + k];
            }
        }
        if (flipped) flipped[i] = fl;
        cd s = 0.0;
        for (int k = 0; k < n; ++k) s += T[(size_t)i * n + k] * cur[(size_t)i * n + k];
        mcur[i] = s;
    }
    // Tv = (conj(Ti)^-1)^T = (conj(Ti)^T)^-1: invert the conjugate transpose; a
    // sign pattern of +-1 rows can be singular, caught by a relative pivot bound
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) K[(size_t)k * n + i] = std::conj(T[(size_t)i * n + k]);
    if (!invert(n, K, 1e-12)) return OPEM_ERR_BREAKDOWN;
    for (int i = 0; i < n; ++i) {
        cd s = 0.0;
        for (int k = 0; k < n; ++k) s += K[(size_t)i * n + k] * vol[(size_t)i * n + k];
        mvol[i] = s;
    }
    for (int i = 0; i < n * n; ++i) {
        Ti[2 * i] = T[i].real(); Ti[2 * i + 1] = T[i].imag();
        Tv[2 * i] = K[i].real(); Tv[2 * i + 1] = K[i].imag();
    }
    for (int i = 0; i < n; ++i) {
        if (Im) { Im[2 * i] = mcur[i].real(); Im[2 * i + 1] = mcur[i].imag(); }
        if (Vm) { Vm[2 * i] = mvol[i].real(); Vm[2 * i + 1] = mvol[i].imag(); }
    }
    return OPEM_OK;
}

// Modal to single-ended conversion, fem3D::build_Mc_Ms with conversion = 0
// (src/OpenParEM3D/fem3D.cpp:1586-1900) and Result::SparameterConversion
// (results.cpp:587-630): S holds the modal S-parameters of the ports' modes
// (S-port order), Zmode their impedances; Tv and Ti map the single-ended line
// voltages / currents of each port to its modal ones (the port's Tv, Ti
// blocks on the diagonal, S-port order).  Kv = Tv^-1, Ki = Ti^-1 take modal to
// single-ended; za = Zmode, zb = zref on every S-port; then term1, term2, Ms,
// Mc and S_b as in the mixed-mode conversion above.
int opem_s_single_ended(int nports, const double* S, const double* Zmode, const double* Tv, const double* Ti,
                        double zref, double* S_out, double* Zo_out) {
    if (nports < 1 || !S || !Zmode || !Tv || !Ti || !(zref > 0) || !S_out) return OPEM_ERR_ARG;
    const int n = nports;
    std::vector<cd> Kv((size_t)n * n), Ki((size_t)n * n), rza(n);
    for (int i = 0; i < n * n; ++i) {
        Kv[i] = cd(Tv[2 * i], Tv[2 * i + 1]);
        Ki[i] = cd(Ti[2 * i], Ti[2 * i + 1]);
    }
    if (!invert(n, Kv) || !invert(n, Ki)) return OPEM_ERR_BREAKDOWN;
    for (int j = 0; j < n; ++j) {
        const cd z(Zmode[2 * j], Zmode[2 * j + 1]);
        if (!(std::abs(z) > 0)) return OPEM_ERR_ARG;
        rza[j] = std::sqrt(z);
    }
    const double rzb = std::sqrt(zref);
    std::vector<cd> Ms((size_t)n * n), Mc((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const cd t1 = Kv[(size_t)i * n + j] * rza[j] / rzb;
            const cd t2 = Ki[(size_t)i * n + j] * rzb / rza[j];
            Ms[(size_t)i * n + j] = 0.5 * (t1 + t2);
            Mc[(size_t)i * n + j] = 0.5 * (t1 - t2);
        }
    std::vector<cd> Sa((size_t)n * n);
    for (int i = 0; i < n * n; ++i) Sa[i] = cd(S[2 * i], S[2 * i + 1]);
    std::vector<cd> num = matmul(n, Ms, Sa), den = matmul(n, Mc, Sa);
    for (int i = 0; i < n * n; ++i) { num[i] += Mc[i]; den[i] += Ms[i]; }
    if (!invert(n, den)) return OPEM_ERR_BREAKDOWN;
    std::vector<cd> Sb = matmul(n, num, den);
    for (int i = 0; i < n * n; ++i) { S_out[2 * i] = Sb[i].real(); S_out[2 * i + 1] = Sb[i].imag(); }
    if (Zo_out)
        for (int i = 0; i < n; ++i) { Zo_out[2 * i] = zref; Zo_out[2 * i + 1] = 0.0; }
    return OPEM_OK;
}

// Touchstone 2.0 (the reference's saveTouchstone branch for mixed-mode data,
// results.cpp:1210-1372): "[Version] 2.0", the option line, "[Number of Ports]",
// "[Two-Port Data Order] 21_12" for two ports, "[Number of Frequencies]",
// "[Matrix Format] Full", "[Mixed-Mode Order]" with S<i> / C<p>,<n> / D<p>,<n>
// when pairs are given, "[Network Data]", the 1.1 data layout, "[End]".
int opem_write_touchstone2(const char* path, int nfreq, const double* freqs, int nports, const double* S,
                           double zref, const char* format, const char* unit, int npairs, const int* pairs) {
    if (!path || nfreq < 1 || !freqs || nports < 1 || !S || !(zref > 0) || !format || !unit || npairs < 0 ||
        (npairs > 0 && !pairs))
        return OPEM_ERR_ARG;
    const std::string fmt(format), un(unit);
    if (fmt != "RI" && fmt != "MA" && fmt != "DB") return OPEM_ERR_ARG;
    const double scale = unit_scale(un);
    if (scale == 0) return OPEM_ERR_ARG;
    const int n = nports;
    std::vector<std::string> info(n), order(n);
    for (int i = 0; i < n; ++i) {
        info[i] = "! S-port S" + std::to_string(i + 1) + " net" + std::to_string(i + 1);
        order[i] = "S" + std::to_string(i + 1);
    }
    for (int k = 0; k < npairs; ++k) {
        const int p = pairs[2 * k], q = pairs[2 * k + 1];
        if (p < 1 || p > n || q < 1 || q > n || p == q) return OPEM_ERR_ARG;
        const std::string nets = "net" + std::to_string(p) + "_net" + std::to_string(q);
        info[p - 1] = "! S-port comm_" + nets;
        info[q - 1] = "! S-port diff_" + nets;
        order[p - 1] = "C" + std::to_string(p) + "," + std::to_string(q);
        order[q - 1] = "D" + std::to_string(p) + "," + std::to_string(q);
    }
    FILE* f = std::fopen(path, "w");
    if (!f) return OPEM_ERR_ARG;
    std::fprintf(f, "! opem-b200\n! %d-port S-parameter data\n", n);
    for (auto& l : info) std::fprintf(f, "%s\n", l.c_str());
    std::fprintf(f, "[Version] 2.0\n# %s S %s R %.15g\n[Number of Ports] %d\n", un.c_str(), fmt.c_str(), zref, n);
    if (n == 2) std::fprintf(f, "[Two-Port Data Order] 21_12\n");
    std::fprintf(f, "[Number of Frequencies] %d\n[Matrix Format] Full\n", nfreq);
    if (npairs > 0) {
        std::fprintf(f, "[Mixed-Mode Order]");
        for (auto& o : order) std::fprintf(f, " %s", o.c_str());
        std::fprintf(f, "\n");
    }
    std::fprintf(f, "[Network Data]\n");
    for (int q = 0; q < nfreq; ++q) write_point(f, n, S + (size_t)2 * n * n * q, freqs[q] * scale, fmt);
    std::fprintf(f, "[End]\n");
    const bool ok = std::ferror(f) == 0;
    std::fclose(f);
    return ok ? OPEM_OK : OPEM_ERR_ARG;
}

int opem_s_renormalize(int nports, const double* S, const double* Zo, double zref_re, double zref_im, double* S_out) {
    if (nports < 1 || nports > 64 || !S || !Zo || !S_out) return OPEM_ERR_ARG;
    const int n = nports;
    const cd zref(zref_re, zref_im);
    if (!(std::abs(zref) > 0)) return OPEM_ERR_ARG;
    std::vector<cd> s((size_t)n * n), k(n);
    for (int i = 0; i < n * n; ++i) s[i] = cd(S[2 * i], S[2 * i + 1]);
    for (int i = 0; i < n; ++i) {
        const cd z(Zo[2 * i], Zo[2 * i + 1]);
        if (!(std::abs(z) > 0)) return OPEM_ERR_ARG;
        k[i] = std::sqrt(z);
    }
    // Z = k (I + S) (I - S)^-1 k
    std::vector<cd> ipS = s, imS((size_t)n * n);
    for (int i = 0; i < n * n; ++i) imS[i] = -s[i];
    for (int i = 0; i < n; ++i) {
        ipS[(size_t)i * n + i] += 1.0;
        imS[(size_t)i * n + i] += 1.0;
    }
    if (!invert(n, imS)) return OPEM_ERR_BREAKDOWN;
    std::vector<cd> Z = matmul(n, ipS, imS);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) Z[(size_t)i * n + j] *= k[i] * k[j];
    // S' = (Z/Zref + I)^-1 (Z/Zref - I)
    std::vector<cd> zp((size_t)n * n), zm((size_t)n * n);
    for (int i = 0; i < n * n; ++i) zp[i] = zm[i] = Z[i] / zref;
    for (int i = 0; i < n; ++i) {
        zp[(size_t)i * n + i] += 1.0;
        zm[(size_t)i * n + i] -= 1.0;
    }
    if (!invert(n, zp)) return OPEM_ERR_BREAKDOWN;
    std::vector<cd> out = matmul(n, zp, zm);
    for (int i = 0; i < n * n; ++i) {
        S_out[2 * i] = out[i].real();
        S_out[2 * i + 1] = out[i].imag();
    }
    return OPEM_OK;
}

int opem_write_touchstone(const char* path, int nfreq, const double* freqs, int nports, const double* S, double zref,
                          const char* format, const char* unit) {
    if (!path || nfreq < 1 || !freqs || nports < 1 || !S || !(zref > 0) || !format || !unit) return OPEM_ERR_ARG;
    const std::string fmt(format), un(unit);
    if (fmt != "RI" && fmt != "MA" && fmt != "DB") return OPEM_ERR_ARG;
    const double scale = unit_scale(un);
    if (scale == 0) return OPEM_ERR_ARG;
    FILE* f = std::fopen(path, "w");
    if (!f) return OPEM_ERR_ARG;
    const int n = nports;
    std::fprintf(f, "! opem-b200\n! %d-port S-parameter data\n", n);
    for (int i = 0; i < n; ++i) std::fprintf(f, "! S-port %d net%d\n", i + 1, i + 1);
    std::fprintf(f, "# %s S %s R %.15g\n", un.c_str(), fmt.c_str(), zref);
    if (n < 3) {
        std::fprintf(f, "!freq");
        const char* h1 = fmt == "RI" ? "ReS" : (fmt == "MA" ? "magS" : "dBS");
        const char* h2 = fmt == "RI" ? "ImS" : "angS";
        for (int col = 0; col < n; ++col)
            for (int row = 0; row < n; ++row) std::fprintf(f, " %s%d%d %s%d%d", h1, row + 1, col + 1, h2, row + 1, col + 1);
        std::fprintf(f, "\n");
    }
    for (int q = 0; q < nfreq; ++q) write_point(f, n, S + (size_t)2 * n * n * q, freqs[q] * scale, fmt);
    const bool ok = std::ferror(f) == 0;
    std::fclose(f);
    return ok ? OPEM_OK : OPEM_ERR_ARG;
}

// Change of S between two adaptive passes (ResultDatabase::
// calculate_maxRelativeError, results.cpp:714-768): the largest column 2-norm of
// S_cur^-1 (S_prev - S_cur).
int opem_s_relative_change(int nports, const double* S_prev, const double* S_cur, double* out) {
    if (nports < 1 || !S_prev || !S_cur || !out) return OPEM_ERR_ARG;
    const int n = nports;
    std::vector<cd> inv((size_t)n * n), d((size_t)n * n);
    for (int i = 0; i < n * n; ++i) {
        inv[i] = cd(S_cur[2 * i], S_cur[2 * i + 1]);
        d[i] = cd(S_prev[2 * i], S_prev[2 * i + 1]) - inv[i];
    }
    if (!invert(n, inv)) return OPEM_ERR_BREAKDOWN;
    const std::vector<cd> e = matmul(n, inv, d);
    double best = 0;
    for (int c = 0; c < n; ++c) {
        double s = 0;
        for (int r = 0; r < n; ++r) s += std::norm(e[(size_t)r * n + c]);
        best = std::max(best, std::sqrt(s));
    }
    *out = best;
    return OPEM_OK;
}

// Results CSV (ResultDatabase::saveCSV, results.cpp:940-1052, and
// Result::saveCSV, :205-230): "#Touchstone format,F", "#frequency unit,U",
// "#number of frequencies,n", "#number of ports,N", one "#S-port i,neti,zref"
// line per port ("not renormalized" for zref <= 0), the column header, then one
// line per frequency.  Values are written in the header's order, S(row;col)
// with the column (driven port) outer and the row (receiving port) inner, which
// is the order the reference's reader and comparator take them in.
int opem_write_results_csv(const char* path, int nfreq, const double* freqs, int nports, const double* S, double zref,
                           const char* format, const char* unit) {
    if (!path || nfreq < 1 || !freqs || nports < 1 || !S || !format || !unit) return OPEM_ERR_ARG;
    const std::string fmt(format), un(unit);
    if (fmt != "RI" && fmt != "MA" && fmt != "DB") return OPEM_ERR_ARG;
    const double scale = unit_scale(un);
    if (scale == 0) return OPEM_ERR_ARG;
    FILE* f = std::fopen(path, "w");
    if (!f) return OPEM_ERR_ARG;
    const int n = nports;
    std::fprintf(f, "#opem-b200\n#Touchstone format,%s\n#frequency unit,%s\n#number of frequencies,%d\n"
                    "#number of ports,%d\n", fmt.c_str(), un.c_str(), nfreq, n);
    for (int i = 0; i < n; ++i) {
        if (zref > 0) std::fprintf(f, "#S-port %d,net%d,%.15g\n", i + 1, i + 1, zref);
        else std::fprintf(f, "#S-port %d,net%d,not renormalized\n", i + 1, i + 1);
    }
    std::fprintf(f, "#Frequency(%s)", un.c_str());
    const char* h1 = fmt == "RI" ? "Re" : (fmt == "MA" ? "mag" : "dB");
    const char* h2 = fmt == "RI" ? "Im" : "deg";
    for (int col = 0; col < n; ++col)
        for (int row = 0; row < n; ++row)
            std::fprintf(f, ",%s(S(%d;%d)),%s(S(%d;%d))", h1, row + 1, col + 1, h2, row + 1, col + 1);
    std::fprintf(f, "\n");
    for (int q = 0; q < nfreq; ++q) {
        const double* Sq = S + (size_t)2 * n * n * q;
        std::fprintf(f, "%.15g", freqs[q] * scale);
        for (int col = 0; col < n; ++col)
            for (int row = 0; row < n; ++row) {
                const cd v(Sq[2 * (row * n + col)], Sq[2 * (row * n + col) + 1]);
                double a, b;
                if (fmt == "RI") { a = v.real(); b = v.imag(); }
                else if (fmt == "MA") { a = std::abs(v); b = std::arg(v) * 180.0 / M_PI; }
                else { a = 20.0 * std::log10(std::abs(v)); b = std::arg(v) * 180.0 / M_PI; }
                std::fprintf(f, ",%.15g,%.15g", a, b);
            }
        std::fprintf(f, "\n");
    }
    const bool ok = std::ferror(f) == 0;
    std::fclose(f);
    return ok ? OPEM_OK : OPEM_ERR_ARG;
}

}  // extern "C"

namespace {

// the reference's frequency match (double_compare, OpenParEMCommon/misc.cpp:76-84)
bool same_value(double a, double b, double tol) {
    if (a == b) return true;
    if (a == 0 && std::fabs(b) < tol) return true;
    if (b == 0 && std::fabs(a) < tol) return true;
    if (std::fabs(a) < tol && std::fabs(b) < tol) return true;
    return std::fabs((a - b) / a) < tol;
}

bool parse_double(const std::string& t, double& v) {
    try {
        size_t k = 0;
        v = std::stod(t, &k);
        return k == t.size() || t.find_first_not_of(" \t\r", k) == std::string::npos;
    } catch (...) {
        return false;
    }
}

bool parse_int(const std::string& t, int& v) {
    double d;
    if (!parse_double(t, d) || d != std::floor(d)) return false;
    v = (int)d;
    return true;
}

struct TestCase {
    std::string name, var, fn;
    double freq = 0, value = 0, tol = 0, found = 0, error = 0;
    int out = 0, in = 0;
    bool passed = false;
};

}  // namespace

extern "C" {

// Regression comparator (process3D, src/OpenParEM3D/process3D.cpp:105-462,
// 481-560): test cases "name,frequency,magS(dB)|argS(deg),portOut,portIn,
// equal|lessthan|greaterthan,expected|threshold[,tolerance]" (after a
// "# ResultDatabase::save_as_test" line; '#' lines and "//" tails are comments)
// evaluated against a results CSV: the first result whose frequency matches to
// 1e-12 relative, magS(dB) / argS(deg) of S(portOut;portIn) (values in the
// CSV's format, converted to dB and degrees; the reference's files are written
// in DB), "equal" as relative error against the tolerance (argS over +-360
// deg), "lessthan" / "greaterthan" against the threshold (argS wrapped into
// (-180, 180)).  The cases are ordered by |error| (equal) or |found value|
// (the others), largest first, by the reference's own exchange procedure, and
// written to out_path in its _test_results.csv layout.  Antenna-metric cases
// (PatternDatabase) are not supported (OPEM_ERR_UNSUPPORTED).
int opem_evaluate_test_cases(const char* test_cases_path, const char* results_csv_path, const char* out_path,
                             int* ncases, int* npassed) {
    if (!test_cases_path || !results_csv_path || !out_path) return OPEM_ERR_ARG;
    std::ifstream tc(test_cases_path);
    if (!tc) return OPEM_ERR_ARG;
    std::vector<TestCase> cases;
    std::string line;
    while (std::getline(tc, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.empty()) continue;
        if (line == "# PatternDatabase::save_as_test") return OPEM_ERR_UNSUPPORTED;
        const size_t first = line.find_first_not_of(" \t");
        if (first == std::string::npos || line[first] == '#') continue;
        line = line.substr(0, line.find("//"));
        std::vector<std::string> v;
        std::stringstream ss(line);
        std::string e;
        while (std::getline(ss, e, ',')) v.push_back(e);
        TestCase c;
        if (v.size() < 7) return OPEM_ERR_ARG;
        c.name = v[0];
        c.var = v[2];
        c.fn = v[5];
        if (!parse_double(v[1], c.freq) || !parse_int(v[3], c.out) || !parse_int(v[4], c.in)) return OPEM_ERR_ARG;
        if (c.var != "magS(dB)" && c.var != "argS(deg)") return OPEM_ERR_ARG;
        if (c.fn != "equal" && c.fn != "lessthan" && c.fn != "greaterthan") return OPEM_ERR_ARG;
        if (v.size() != (c.fn == "equal" ? 8u : 7u)) return OPEM_ERR_ARG;
        if (!parse_double(v[6], c.value)) return OPEM_ERR_ARG;
        if (c.fn == "equal" && !parse_double(v[7], c.tol)) return OPEM_ERR_ARG;
        cases.push_back(c);
    }
    // results CSV
    std::ifstream rc(results_csv_path);
    if (!rc) return OPEM_ERR_ARG;
    std::string fmt = "DB", unit = "Hz";
    int N = 0;
    std::vector<std::pair<double, std::vector<cd>>> results;   // frequency, (value pairs in file order)
    while (std::getline(rc, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.empty()) continue;
        std::vector<std::string> v;
        std::stringstream ss(line);
        std::string e;
        while (std::getline(ss, e, ',')) v.push_back(e);
        if (line[0] == '#') {
            if (v.size() >= 2 && v[0] == "#Touchstone format") fmt = v[1];
            if (v.size() >= 2 && v[0] == "#frequency unit") unit = v[1];
            if (v.size() >= 2 && v[0] == "#number of ports" && !parse_int(v[1], N)) return OPEM_ERR_ARG;
            continue;
        }
        const double sc = unit_scale(unit);
        if (sc == 0 || N < 1 || v.size() != (size_t)(1 + 2 * N * N)) return OPEM_ERR_ARG;
        double f;
        if (!parse_double(v[0], f)) return OPEM_ERR_ARG;
        std::vector<cd> vals(N * N);
        for (int k = 0; k < N * N; ++k) {
            double a, b;
            if (!parse_double(v[1 + 2 * k], a) || !parse_double(v[2 + 2 * k], b)) return OPEM_ERR_ARG;
            vals[k] = cd(a, b);
        }
        results.push_back({f / sc, vals});
    }
    // evaluation
    int np = 0;
    for (TestCase& c : cases) {
        c.passed = false;
        c.found = 0;
        const std::vector<cd>* R = nullptr;
        for (auto& r : results)
            if (same_value(r.first, c.freq, 1e-12)) { R = &r.second; break; }
        if (R && c.out >= 1 && c.out <= N && c.in >= 1 && c.in <= N) {
            // pair k = (portIn - 1) N + (portOut - 1): the driven port outer, as the header orders S(row;col)
            const cd pr = (*R)[(c.in - 1) * N + (c.out - 1)];
            double db = pr.real(), deg = pr.imag();
            if (fmt == "RI") { db = 20 * std::log10(std::abs(pr)); deg = std::arg(pr) * 180 / M_PI; }
            if (fmt == "MA") { db = 20 * std::log10(pr.real()); }
            if (c.var == "magS(dB)") {
                c.found = db;
                if (c.fn == "equal") {
                    c.error = c.value == 0 ? std::fabs(c.found) : std::fabs((c.found - c.value) / c.value);
                    c.passed = c.error <= c.tol;
                } else if (c.fn == "lessthan") c.passed = c.found <= c.value;
                else c.passed = c.found >= c.value;
            } else {
                c.found = deg;
                if (c.fn == "equal") {
                    if (c.value == 0) c.error = std::fabs(c.found);
                    else {
                        const double e1 = std::fabs((c.found - c.value) / c.value);
                        const double e2 = std::fabs((c.found + 360 - c.value) / c.value);
                        const double e3 = std::fabs((c.found - 360 - c.value) / c.value);
                        c.error = std::min(std::min(e1, e2), e3);
                    }
                    c.passed = c.error <= c.tol;
                } else {
                    while (c.found >= 180) c.found -= 360;
                    while (c.found <= -180) c.found += 360;
                    c.passed = c.fn == "lessthan" ? c.found <= c.value : c.found >= c.value;
                }
            }
        }
        if (c.passed) ++np;
    }
    // the reference's ordering (TestCaseDatabase::sort, process3D.cpp:390-422)
    const size_t n = cases.size();
    auto key = [&](size_t k) { return std::fabs(cases[k].fn == "equal" ? cases[k].error : cases[k].found); };
    std::vector<size_t> idx(n);
    for (size_t i = 0; i < n; ++i) idx[i] = i;
    for (size_t i = 0; i + 1 < n; ++i) {
        bool found = true;
        while (found) {
            found = false;
            for (size_t j = i + 1; j < n; ++j)
                if (key(idx[i]) < key(idx[j])) {
                    found = true;
                    std::swap(idx[i], idx[j]);
                }
        }
    }
    FILE* f = std::fopen(out_path, "w");
    if (!f) return OPEM_ERR_ARG;
    std::fprintf(f, "# name,status,frequency,portOut,portIn,testVariable,testFunction,[equal:expectedValue,]"
                    "foundValue,[equal:error,tolerance | lessthan:threshold | greaterthan:threshold\n");
    for (size_t k : idx) {
        const TestCase& c = cases[k];
        std::fprintf(f, "%s,%s,%.15g,%d,%d,%s,%s,", c.name.c_str(), c.passed ? "pass" : "FAIL", c.freq, c.out, c.in,
                     c.var.c_str(), c.fn.c_str());
        if (c.fn == "equal") std::fprintf(f, "%.15g,", c.value);
        std::fprintf(f, "%.15g,", c.found);
        if (c.fn == "equal") std::fprintf(f, "%.15g,%.15g,\n", c.error, c.tol);
        else std::fprintf(f, "%.15g,\n", c.value);
    }
    const bool ok = std::ferror(f) == 0;
    std::fclose(f);
    if (ncases) *ncases = (int)n;
    if (npassed) *npassed = np;
    return ok ? OPEM_OK : OPEM_ERR_ARG;
}

}  // extern "C"
