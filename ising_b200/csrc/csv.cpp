// csv.cpp -- the reference's CSV outputs, written byte-for-byte in its Fortran formats.
//
// Edit descriptors follow the Fortran 2008 rules as gfortran applies them: F0.d writes the
// minimal width and omits the optional zero before the point (unified-analysis.py:234-247
// strips it when rebuilding file names), E0.d writes a 0.ddd mantissa with an exponent of
// minimal digits (unified-analysis.py:178-199), ESw.d right-justifies one digit before the
// point with a two-digit exponent, Iw.m pads to m digits.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace isg {
namespace fmt {

std::string F0(double x, int d) {
    if (std::isnan(x)) return "NaN";
    if (std::isinf(x)) return x > 0 ? "Infinity" : "-Infinity";
    char buf[512];
    std::snprintf(buf, sizeof buf, "%.*f", d, std::fabs(x));
    const char* s = buf;
    if (s[0] == '0' && s[1] == '.') ++s;
    std::string out = std::signbit(x) ? "-" : "";
    out += s;
    return out;
}

std::string I0m(long v, int m) {
    char buf[64];
    if (v < 0) std::snprintf(buf, sizeof buf, "-%0*ld", m, -v);
    else std::snprintf(buf, sizeof buf, "%0*ld", m, v);
    return buf;
}

std::string ES(double x, int w, int d) {
    std::string out;
    if (std::isnan(x)) out = "NaN";
    else {
        char buf[128];
        std::snprintf(buf, sizeof buf, "%.*e", d, x);
        char* e = std::strchr(buf, 'e');
        const int ex = std::atoi(e + 1);
        *e = 0;
        char tail[16];
        if (ex > 99 || ex < -99) std::snprintf(tail, sizeof tail, "%+04d", ex);
        else std::snprintf(tail, sizeof tail, "E%+03d", ex);
        out = std::string(buf) + tail;
    }
    if ((int)out.size() > w) return std::string(w, '*');
    return std::string(w - out.size(), ' ') + out;
}

std::string E0(double x, int d) {
    if (x == 0.0) return "0." + std::string(d, '0') + "E+0";
    char buf[128];
    std::snprintf(buf, sizeof buf, "%.*e", d - 1, std::fabs(x));
    char* e = std::strchr(buf, 'e');
    const int ex = std::atoi(e + 1) + 1;
    *e = 0;
    std::string mant = "0.";
    mant += buf[0];
    mant += (buf + 2);
    char tail[16];
    std::snprintf(tail, sizeof tail, "E%+d", ex);
    return (x < 0 ? "-" : "") + mant + tail;
}

}  // namespace fmt
}  // namespace isg

using namespace isg;

namespace {
int write_all(const char* path, const std::string& s, bool append) {
    FILE* f = std::fopen(path, append ? "ab" : "wb");
    if (!f) return fail(ISING_ERR_ARG, std::string("cannot open ") + path);
    const size_t n = std::fwrite(s.data(), 1, s.size(), f);
    const int cl = std::fclose(f);
    if (n != s.size() || cl != 0) return fail(ISING_ERR_ARG, std::string("short write to ") + path);
    return ISING_OK;
}
}  // namespace

// write_spins_to_file (src/LLG.f90:93-172)
extern "C" int ising_write_spins_csv(const ising_mesh* m, int replica, const char* path, int append,
                                     int include_header, int frame_index) {
    if (!m || !path) return fail(ISING_ERR_ARG, "NULL argument");
    const int64_t N = m->lat.natoms;
    std::vector<double> s((size_t)3 * N);
    int st = ising_spins_get(m, replica, s.data());
    if (st != ISING_OK) return st;
    for (int64_t i = 0; i < 3 * N; ++i)
        if (std::isnan(s[i])) return fail(ISING_ERR_NAN, "NaN value encountered");   // :104-109
    std::string out;
    out.reserve((size_t)N * 140 + 64);
    if (frame_index >= 0) out += "# Frame: " + std::to_string(frame_index) + "\n";    // :131-139
    if (include_header) out += "x,y,z,Sx,Sy,Sz\n";                                  // :142-149
    float p[3];
    for (int64_t i = 0; i < N; ++i) {                                               // :152-166
        m->lat.position(i, p);
        out += fmt::ES((double)p[0], 22, 14); out += ',';
        out += fmt::ES((double)p[1], 22, 14); out += ',';
        out += fmt::ES((double)p[2], 22, 14); out += ',';
        out += fmt::ES(s[i], 22, 14); out += ',';
        out += fmt::ES(s[N + i], 22, 14); out += ',';
        out += fmt::ES(s[2 * N + i], 22, 14); out += '\n';
    }
    return write_all(path, out, append != 0);
}

// data_<tag>.csv record (src/PT.f90:318-331,358-362): header line, then the trimmed
// "J,D,B,T," buffer followed by the untrimmed 500-character statistics buffer, a new_line
// and the record terminator of write(...,'(A)').
extern "C" int ising_write_pt_data_csv(const char* path, double J, double D, double B, double T, double wnd_mid,
                                       int sk_mid, double wnd_spread, const double m[3]) {
    if (!path || !m) return fail(ISING_ERR_ARG, "NULL argument");
    std::string out = "J,D,B,T,winding_number_middle,skyrmion_number_middle,winding_number_spread,sx,sy,sz\n";
    out += fmt::F0(J, 4) + "," + fmt::F0(D, 4) + "," + fmt::F0(B, 4) + "," + fmt::F0(T, 10) + ",";
    std::string b2 = fmt::F0(wnd_mid, 4) + "," + fmt::I0m(sk_mid, 4) + "," + fmt::F0(wnd_spread, 2) + "," +
                     fmt::F0(m[0], 2) + "," + fmt::F0(m[1], 2) + "," + fmt::F0(m[2], 2);
    if (b2.size() < 500) b2 += std::string(500 - b2.size(), ' ');
    out += b2 + "\n\n";
    return write_all(path, out, false);
}

// (F0.4,"_",F0.4,"_",F0.4,"_",e0.4) of src/PT.f90:337-338
extern "C" int ising_pt_file_tag(char* buf, size_t cap, double J, double D, double B, double T) {
    if (!buf) return fail(ISING_ERR_ARG, "NULL buffer");
    const std::string s = fmt::F0(J, 4) + "_" + fmt::F0(D, 4) + "_" + fmt::F0(B, 4) + "_" + fmt::E0(T, 4);
    if (s.size() + 1 > cap) return fail(ISING_ERR_ARG, "buffer too small");
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return ISING_OK;
}

// write_winding_number_density (rsp:544-580): every record is "x,y,z,d" + new_line written
// into the buffer, trimmed, plus another new_line; the final write adds a terminator.
extern "C" int ising_write_winding_density_csv(const ising_mesh* m, int replica, const char* path) {
    if (!m || !path) return fail(ISING_ERR_ARG, "NULL argument");
    const Lattice& L = m->lat;
    std::vector<double> dens((size_t)L.nx * L.ny);
    std::string out = "x,y,z,Winding_Density\n";
    for (int i = 1; i <= L.nz; ++i) {
        int st = ising_winding_density(m, replica, i, dens.data());
        if (st != ISING_OK) return st;
        for (int j = 1; j <= L.nx; ++j)
            for (int k = 1; k <= L.ny; ++k) {
                double pos[3];
                for (int q = 0; q < 3; ++q) pos[q] = ((double)j * L.av[q] + (double)k * L.bv[q]) + (double)i * L.cv[q];
                out += fmt::F0(pos[0], 8) + "," + fmt::F0(pos[1], 8) + "," + fmt::F0(pos[2], 8) + "," +
                       fmt::F0(dens[(j - 1) + (size_t)(k - 1) * L.nx], 8) + "\n\n";
            }
    }
    out += "\n";
    return write_all(path, out, false);
}
