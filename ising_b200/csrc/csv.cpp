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
#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace isg {
namespace fmt {

// F0.d appended to o without a temporary string
void F0_app(std::string& o, double x, int d) {
    if (std::isnan(x)) { o += "NaN"; return; }
    if (std::isinf(x)) { o += x > 0 ? "Infinity" : "-Infinity"; return; }
    char buf[512];
    std::snprintf(buf, sizeof buf, "%.*f", d, std::fabs(x));
    const char* s = buf;
    if (s[0] == '0' && s[1] == '.') ++s;
    if (std::signbit(x)) o += '-';
    o += s;
}

std::string F0(double x, int d) {
    std::string out;
    F0_app(out, x, d);
    return out;
}

// Fw.d appended to o: right-justified in w characters (the zero before the point written, as
// it is whenever the field has room), w asterisks when the number does not fit
void Fw_app(std::string& o, double x, int w, int d) {
    char buf[512];
    const int n = std::snprintf(buf, sizeof buf, "%*.*f", w, d, x);
    if (n > w || std::isnan(x) || std::isinf(x)) { o.append((size_t)w, '*'); return; }
    o.append(buf, (size_t)n);
}

std::string I0m(long v, int m) {
    char buf[64];
    if (v < 0) std::snprintf(buf, sizeof buf, "-%0*ld", m, -v);
    else std::snprintf(buf, sizeof buf, "%0*ld", m, v);
    return buf;
}

// ESw.d appended to o: the field is built in a stack buffer and right-justified in place
void ES_app(std::string& o, double x, int w, int d) {
    char buf[160];
    int n;
    if (std::isnan(x)) {
        std::memcpy(buf, "NaN", 4);
        n = 3;
    } else {
        n = std::snprintf(buf, sizeof buf - 8, "%.*e", d, x);
        char* e = std::strchr(buf, 'e');
        const int ex = std::atoi(e + 1);
        if (ex > 99 || ex < -99) n = (int)(e - buf) + std::snprintf(e, 8, "%+04d", ex);
        else n = (int)(e - buf) + std::snprintf(e, 8, "E%+03d", ex);
    }
    if (n > w) { o.append((size_t)w, '*'); return; }
    o.append((size_t)(w - n), ' ');
    o.append(buf, (size_t)n);
}

std::string ES(double x, int w, int d) {
    std::string out;
    ES_app(out, x, w, d);
    return out;
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
int write_parts(const char* path, const std::vector<std::string>& parts, bool append) {
    FILE* f = std::fopen(path, append ? "ab" : "wb");
    if (!f) return fail(ISING_ERR_ARG, std::string("cannot open ") + path);
    bool ok = true;
    for (const std::string& s : parts) ok = ok && std::fwrite(s.data(), 1, s.size(), f) == s.size();
    const int cl = std::fclose(f);
    if (!ok || cl != 0) return fail(ISING_ERR_ARG, std::string("short write to ") + path);
    return ISING_OK;
}

int write_all(const char* path, const std::string& s, bool append) {
    return write_parts(path, std::vector<std::string>{s}, append);
}

// Formats records [0, n) in contiguous ranges on all host threads: fn(i, out) appends record i
// to its thread's buffer.  The buffers, written in order, are the sequential output; the
// reference builds the same text by repeated concatenation (rsp:533,573), O(n^2).
template <typename Fn>
std::vector<std::string> format_records(int64_t n, size_t bytes_per_record, const Fn& fn) {
    const int64_t per_thread_min = 4096;
    const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(hw, n / per_thread_min));
    std::vector<std::string> parts(nt);
    auto work = [&](int t) {
        const int64_t a = n * t / nt, b = n * (t + 1) / nt;
        std::string& o = parts[t];
        o.reserve((size_t)(b - a) * bytes_per_record);
        for (int64_t i = a; i < b; ++i) fn(i, o);
    };
    std::vector<std::thread> pool;
    pool.reserve(nt - 1);
    for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
    work(0);
    for (std::thread& th : pool) th.join();
    return parts;
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
    std::string head;
    if (frame_index >= 0) head += "# Frame: " + std::to_string(frame_index) + "\n";   // :131-139
    if (include_header) head += "x,y,z,Sx,Sy,Sz\n";                                 // :142-149
    const Lattice& L = m->lat;
    std::vector<std::string> parts = format_records(N, 6 * 23, [&](int64_t i, std::string& o) {  // :152-166
        float p[3];
        L.position(i, p);
        fmt::ES_app(o, (double)p[0], 22, 14); o += ',';
        fmt::ES_app(o, (double)p[1], 22, 14); o += ',';
        fmt::ES_app(o, (double)p[2], 22, 14); o += ',';
        fmt::ES_app(o, s[i], 22, 14); o += ',';
        fmt::ES_app(o, s[N + i], 22, 14); o += ',';
        fmt::ES_app(o, s[2 * N + i], 22, 14); o += '\n';
    });
    parts.insert(parts.begin(), head);
    return write_parts(path, parts, append != 0);
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

// write(frame_filename, '(A,A,I5.5,A)') trim(output_dir), "/frame_", index, ".csv"
// (src/ISING.f90:218): five digits with leading zeros, ***** when the value does not fit.
extern "C" int ising_frame_filename(char* buf, size_t cap, const char* output_dir, int index) {
    if (!buf || !output_dir) return fail(ISING_ERR_ARG, "NULL argument");
    std::string dir(output_dir);
    while (!dir.empty() && dir.back() == ' ') dir.pop_back();   // trim()
    // I5.5 needs five digits, so a negative value (which also needs its sign) does not fit
    const std::string num = (index < 0 || index > 99999) ? std::string("*****") : fmt::I0m(index, 5);
    const std::string s = dir + "/frame_" + num + ".csv";
    if (s.size() + 1 > cap) return fail(ISING_ERR_ARG, "buffer too small");
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return ISING_OK;
}

// info.txt of the annealing driver (src/ISING.f90:232-237): the frame count, then numCellsX and
// the default-real lattice parameter, list-directed: blank-separated, integers right-aligned in
// 12 columns and the real with 9 significant digits.  The visualisation scripts read the two
// lines with strip() and split() (skyrmion_evolution_simple.py:86-91, visualise_skyrmion.py:15-20).
extern "C" int ising_write_frame_info(const char* path, int num_frames, int num_cells_x, float lattice_param) {
    if (!path) return fail(ISING_ERR_ARG, "NULL argument");
    char a[64], b[96];
    std::snprintf(a, sizeof a, "%12d\n", num_frames);
    const double v = (double)lattice_param;
    const double av = std::fabs(v);
    char r[48];
    if (av != 0.0 && (av < 0.1 || av >= 1e8)) std::snprintf(r, sizeof r, "%.8E", v);
    else std::snprintf(r, sizeof r, "%.*f", av == 0.0 ? 8 : 8 - (int)std::floor(std::log10(av)), v);
    std::snprintf(b, sizeof b, "%12d   %s\n", num_cells_x, r);
    return write_all(path, std::string(a) + b, false);
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
// into the buffer, trimmed, plus another new_line; the final write adds a terminator.  Record
// order is slice i, then j over x, then k over y; the densities of all slices come from one
// device pass.
extern "C" int ising_write_winding_density_csv(const ising_mesh* m, int replica, const char* path) {
    if (!m || !path) return fail(ISING_ERR_ARG, "NULL argument");
    const Lattice& L = m->lat;
    const int64_t plane = (int64_t)L.nx * L.ny;
    std::vector<double> dens((size_t)(plane * L.nz));
    int st = ising_winding_density_all(m, replica, dens.data());
    if (st != ISING_OK) return st;
    std::vector<std::string> parts = format_records(plane * L.nz, 4 * 14, [&](int64_t r, std::string& o) {
        const int i = (int)(r / plane) + 1;
        const int64_t q = r % plane;
        const int j = (int)(q / L.ny) + 1, k = (int)(q % L.ny) + 1;
        double pos[3];
        for (int c = 0; c < 3; ++c) pos[c] = ((double)j * L.av[c] + (double)k * L.bv[c]) + (double)i * L.cv[c];
        fmt::F0_app(o, pos[0], 8); o += ',';
        fmt::F0_app(o, pos[1], 8); o += ',';
        fmt::F0_app(o, pos[2], 8); o += ',';
        fmt::F0_app(o, dens[(size_t)((i - 1) * plane + (j - 1) + (int64_t)(k - 1) * L.nx)], 8);
        o += "\n\n";
    });
    parts.insert(parts.begin(), std::string("x,y,z,Winding_Density\n"));
    parts.push_back("\n");
    return write_parts(path, parts, false);
}

// write_demagnetisation_field_to_file (src/energyMin.f90:559-583): header x,y,z,fx,fy,fz, one
// record per atom with the single-precision position makeChainMesh stores and the field
// components, each F8.4.
extern "C" int ising_write_demag_csv(const ising_mesh* m, int replica, const char* path) {
    if (!m || !path) return fail(ISING_ERR_ARG, "NULL argument");
    const Lattice& L = m->lat;
    const int64_t N = L.natoms;
    std::vector<double> H((size_t)(3 * N));
    int st = ising_demag_field(m, replica, H.data());
    if (st != ISING_OK) return st;
    std::vector<std::string> parts = format_records(N, 6 * 9, [&](int64_t a, std::string& o) {
        float p[3];
        L.position(a, p);
        fmt::Fw_app(o, (double)p[0], 8, 4); o += ',';
        fmt::Fw_app(o, (double)p[1], 8, 4); o += ',';
        fmt::Fw_app(o, (double)p[2], 8, 4); o += ',';
        fmt::Fw_app(o, H[(size_t)a], 8, 4); o += ',';
        fmt::Fw_app(o, H[(size_t)(N + a)], 8, 4); o += ',';
        fmt::Fw_app(o, H[(size_t)(2 * N + a)], 8, 4);
        o += '\n';
    });
    parts.insert(parts.begin(), std::string("x,y,z,fx,fy,fz\n"));
    return write_parts(path, parts, false);
}

// write_winding_number_density_interpolated (rsp:502-540): the same records as
// write_winding_number_density over the (sclx nx) x (scly ny) fine grid of every slice; the
// position of record (j, k) of slice i is j a + k b + i c with the FINE indices j, k, as in the
// reference.
extern "C" int ising_write_winding_density_interpolated_csv(const ising_mesh* m, int replica, const char* path) {
    if (!m || !path) return fail(ISING_ERR_ARG, "NULL argument");
    const Lattice& L = m->lat;
    int sx = 0, sy = 0;
    int st = ising_mesh_interpolation_scale(m, &sx, &sy);
    if (st != ISING_OK) return st;
    const int fx = L.nx * sx, fy = L.ny * sy;
    const int64_t plane = (int64_t)fx * fy;
    std::vector<double> dens((size_t)plane);
    std::vector<std::string> parts;
    parts.emplace_back("x,y,z,Winding_Density\n");
    for (int i = 1; i <= L.nz; ++i) {
        st = ising_winding_density_interpolated(m, replica, i, dens.data());
        if (st != ISING_OK) return st;
        std::vector<std::string> slice = format_records(plane, 4 * 14, [&](int64_t r, std::string& o) {
            const int j = (int)(r / fy) + 1, k = (int)(r % fy) + 1;
            double pos[3];
            for (int c = 0; c < 3; ++c) pos[c] = ((double)j * L.av[c] + (double)k * L.bv[c]) + (double)i * L.cv[c];
            fmt::F0_app(o, pos[0], 8); o += ',';
            fmt::F0_app(o, pos[1], 8); o += ',';
            fmt::F0_app(o, pos[2], 8); o += ',';
            fmt::F0_app(o, dens[(size_t)((j - 1) + (int64_t)(k - 1) * fx)], 8);
            o += "\n\n";
        });
        for (auto& x : slice) parts.push_back(std::move(x));
    }
    parts.push_back("\n");
    return write_parts(path, parts, false);
}
