// Host-side helpers shared by the FP64 and FP32 orchestration: the halo-padded grid on the host,
// the velocity halo rules used by vel_copy! when a dimension is smaller than its halo, and Julia's
// shortest round-trip Float64 formatting for error messages.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pib200.h"

namespace pih {

struct HostGrid {
    int Nx, Ny, Nz, Hx, Hy, Hz, Gx, Gy, Gz;
    int topo[3];
    double dx, dy;
    std::vector<double> dzF, dzC;
    std::vector<uint8_t> lm;
    long long G;
    size_t id(long i, long j, long k) const {
        return (size_t)(i - 1) + (size_t)Gx * ((size_t)(j - 1) + (size_t)Gy * (size_t)(k - 1));
    }
};

// Host halo rules for velocities (HaloRegions/halo_regions.jl:2-99), used by vel_copy!.
// mode 0 tracer rule, 1 velocity rule on the high face.
inline void host_fill_face(const HostGrid& g, std::vector<double>& c, int axis, int face, int mode) {
    int N = axis == 0 ? g.Nx : axis == 1 ? g.Ny : g.Nz;
    int H = axis == 0 ? g.Hx : axis == 1 ? g.Hy : g.Hz;
    int topo = g.topo[axis];
    int n1 = axis == 0 ? g.Gy : g.Gx, n2 = axis == 2 ? g.Gy : g.Gz;
    std::vector<long> dst, src;
    if (face == 0) {
        for (int h = 1; h <= H; ++h) { dst.push_back(h); src.push_back(topo == PI_PERIODIC ? N + h : H + 1); }
    } else if (mode == 1 && topo == PI_BOUNDED) {
        for (int h = N + H + 2; h <= N + 2 * H; ++h) { dst.push_back(h); src.push_back(N + H + 1); }
    } else {
        for (int h = 1; h <= H; ++h) { dst.push_back(N + H + h); src.push_back(topo == PI_PERIODIC ? H + h : N + H); }
    }
    std::vector<double> tmp(dst.size());
    for (int b2 = 1; b2 <= n2; ++b2)
        for (int b1 = 1; b1 <= n1; ++b1) {
            auto at = [&](long a) -> double& {
                if (axis == 0) return c[g.id(a, b1, b2)];
                if (axis == 1) return c[g.id(b1, a, b2)];
                return c[g.id(b1, b2, a)];
            };
            for (size_t q = 0; q < dst.size(); ++q) tmp[q] = at(src[q]);
            for (size_t q = 0; q < dst.size(); ++q) at(dst[q]) = tmp[q];
        }
}

inline void host_fill_halo_vel(const HostGrid& g, std::vector<double>& u, std::vector<double>& v, std::vector<double>& w) {
    host_fill_face(g, u, 0, 1, 1); host_fill_face(g, u, 0, 0, 0);
    host_fill_face(g, u, 1, 0, 0); host_fill_face(g, u, 1, 1, 0);
    host_fill_face(g, u, 2, 0, 0); host_fill_face(g, u, 2, 1, 0);
    host_fill_face(g, v, 1, 1, 1); host_fill_face(g, v, 0, 0, 0); host_fill_face(g, v, 0, 1, 0);
    host_fill_face(g, v, 1, 0, 0); host_fill_face(g, v, 2, 0, 0); host_fill_face(g, v, 2, 1, 0);
    host_fill_face(g, w, 2, 1, 1); host_fill_face(g, w, 0, 0, 0); host_fill_face(g, w, 0, 1, 0);
    host_fill_face(g, w, 1, 0, 0); host_fill_face(g, w, 1, 1, 0); host_fill_face(g, w, 2, 0, 0);
}

// Interior velocity snapshot (reference array layout) → halo-padded fields (vel_copy!).
inline void host_vel_copy(const HostGrid& g, const double* u, const double* v, const double* w,
                   std::vector<double>& U, std::vector<double>& V, std::vector<double>& W) {
    U.assign(g.G, 0.0); V.assign(g.G, 0.0); W.assign(g.G, 0.0);
    int ex = g.topo[0] == PI_BOUNDED, ey = g.topo[1] == PI_BOUNDED, ez = g.topo[2] == PI_BOUNDED;
    auto copy_in = [&](std::vector<double>& f, const double* s, int nx, int ny, int nz) {
        for (int k = 1; k <= nz; ++k) for (int j = 1; j <= ny; ++j) for (int i = 1; i <= nx; ++i)
            f[g.id(i + g.Hx, j + g.Hy, k + g.Hz)] =
                s[(size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)ny * (size_t)(k - 1))];
    };
    copy_in(U, u, g.Nx + ex, g.Ny, g.Nz);
    copy_in(V, v, g.Nx, g.Ny + ey, g.Nz);
    copy_in(W, w, g.Nx, g.Ny, g.Nz + ez);
    host_fill_halo_vel(g, U, V, W);
}

// Julia's string(x::Float64) for the capacity message: shortest round-trip digits.
inline std::string julia_float(double x) {
    char buf[64];
    for (int p = 1; p <= 17; ++p) {
        snprintf(buf, sizeof buf, "%.*g", p, x);
        if (strtod(buf, nullptr) == x) break;
    }
    std::string s(buf);
    size_t e = s.find('e');
    if (e == std::string::npos) {
        if (s.find('.') == std::string::npos && s.find("inf") == std::string::npos && s.find("nan") == std::string::npos) s += ".0";
        return s;
    }
    std::string mant = s.substr(0, e), ex = s.substr(e + 1);
    if (mant.find('.') == std::string::npos) mant += ".0";
    int ev = atoi(ex.c_str());
    return mant + "e" + std::to_string(ev);
}


// Tracer names in the reference's order (src/Biogeochemistry/Biogeochemistry.jl:20).
inline const char* tracer_name(int n) {
    static const char* names[PI_NTRACERS] = { "DIC", "NH4", "NO3", "PO4", "DFe", "DOC", "DON", "DOP",
                                              "PFe_inorg", "POC", "PON", "POP", "PFe_bio", "Dust" };
    return n >= 0 && n < PI_NTRACERS ? names[n] : "?";
}

}  // namespace pih
