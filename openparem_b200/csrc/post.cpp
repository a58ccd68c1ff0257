// S-parameter post-processing on the host: renormalisation to a reference
// impedance and Touchstone 1.1 output (the reference's Result::S2Z / Z2S /
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

}  // namespace

extern "C" {

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
    double scale = 0;
    if (un == "Hz") scale = 1;
    if (un == "kHz") scale = 1e-3;
    if (un == "MHz") scale = 1e-6;
    if (un == "GHz") scale = 1e-9;
    if (scale == 0) return OPEM_ERR_ARG;
    FILE* f = std::fopen(path, "w");
    if (!f) return OPEM_ERR_ARG;
    const int n = nports;
    std::fprintf(f, "! opem-b200\n! %d-port S-parameter data\n", n);
    for (int i = 0; i < n; ++i) std::fprintf(f, "! S-port %d net%d\n", i + 1, i + 1);
    std::fprintf(f, "# %s S %s R %.15g\n", un.c_str(), fmt.c_str(), zref);
    auto pair = [&](const cd& v) {
        double a, b;
        if (fmt == "RI") { a = v.real(); b = v.imag(); }
        else if (fmt == "MA") { a = std::abs(v); b = std::arg(v) * 180.0 / M_PI; }
        else { a = 20.0 * std::log10(std::abs(v)); b = std::arg(v) * 180.0 / M_PI; }
        std::fprintf(f, " %.15g %.15g", a, b);
    };
    if (n < 3) {
        std::fprintf(f, "!freq");
        const char* h1 = fmt == "RI" ? "ReS" : (fmt == "MA" ? "magS" : "dBS");
        const char* h2 = fmt == "RI" ? "ImS" : "angS";
        for (int col = 0; col < n; ++col)
            for (int row = 0; row < n; ++row) std::fprintf(f, " %s%d%d %s%d%d", h1, row + 1, col + 1, h2, row + 1, col + 1);
        std::fprintf(f, "\n");
    }
    for (int q = 0; q < nfreq; ++q) {
        const double* Sq = S + (size_t)2 * n * n * q;
        auto at = [&](int r, int c) { return cd(Sq[2 * (r * n + c)], Sq[2 * (r * n + c) + 1]); };
        std::fprintf(f, "%.15g", freqs[q] * scale);
        if (n < 3) {
            for (int col = 0; col < n; ++col)
                for (int row = 0; row < n; ++row) pair(at(row, col));
            std::fprintf(f, "\n");
        } else {
            for (int row = 0; row < n; ++row) {
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
    }
    const bool ok = std::ferror(f) == 0;
    std::fclose(f);
    return ok ? OPEM_OK : OPEM_ERR_ARG;
}

}  // extern "C"
