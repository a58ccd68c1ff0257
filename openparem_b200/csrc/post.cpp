// S-parameter post-processing on the host: renormalisation to a reference
// impedance, mixed-mode conversion, and Touchstone 1.1 / 2.0 output (the reference's Result::S2Z / Z2S /
// renormalize, src/OpenParEM3D/results.cpp:455-580, and
// ResultDatabase::saveTouchstone, results.cpp:1055-1208).  The file layout
// follows the Touchstone 1.1 conventions the reference writes: "# <unit> S
// <RI|MA|DB> R <Zref>", 1- and 2-port data with S11 S21 S12 S22 (column by
// column) on one line per frequency, more ports row by row with at most four
// pairs per line and a "!row i" comment, 15 significant digits.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/opem_b200.h"

namespace {

using cd = std::complex<double>;

// inverse of an n x n complex matrix (row-major) by Gauss-Jordan with partial pivoting
bool invert(int n, std::vector<cd>& a) {
    std::vector<cd> inv((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r)
            if (std::abs(a[(size_t)r * n + c]) > std::abs(a[(size_t)p * n + c])) p = r;
        if (!(std::abs(a[(size_t)p * n + c]) > 0)) return false;
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

}  // extern "C"
