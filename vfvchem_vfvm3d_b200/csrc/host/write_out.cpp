// Field output in the reference's formats (host). The layout of every file, element for element,
// follows src/base/write_vtu.rs and src/base/write_csv.rs: those files are read by other tools, so the
// bytes must match. Numbers are written as Rust's `{:.9}` prints an f64: fixed notation, 9
// decimals, exact decimal rounding with ties to even (as glibc's "%.9f"), and "NaN", "inf", "-inf".
// Large files are formatted in parallel (OpenMP), in chunks of lines written in order.
#include "write_out.hpp"

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <omp.h>
#include <vector>

namespace vfv {

namespace {

void put_num(std::string& s, double x) {
    if (std::isnan(x)) {
        s += "NaN";
        return;
    }
    if (std::isinf(x)) {
        s += x > 0 ? "inf" : "-inf";
        return;
    }
    char buf[400];  // %.9f of the largest double: 309 integer digits, sign, point, 9 decimals
    const int k = std::snprintf(buf, sizeof buf, "%.9f", x);
    s.append(buf, (size_t)k);
}

void put_int(std::string& s, int64_t v) {
    char buf[24];
    const int k = std::snprintf(buf, sizeof buf, "%lld", (long long)v);
    s.append(buf, (size_t)k);
}

struct File {
    FILE* f = nullptr;
    std::string path, err;
    explicit File(const char* p) : path(p ? p : "") {
        f = p ? std::fopen(p, "wb") : nullptr;
        if (!f) err = "cannot write file '" + path + "': " + (p ? std::strerror(errno) : "no path");
    }
    ~File() {
        if (f) std::fclose(f);
    }
    void put(const std::string& s) {
        if (err.empty() && std::fwrite(s.data(), 1, s.size(), f) != s.size()) err = "cannot write file '" + path + "': " + std::strerror(errno);
    }
    std::string close() {
        if (f && std::fclose(f) != 0 && err.empty()) err = "cannot write file '" + path + "': " + std::strerror(errno);
        f = nullptr;
        return err;
    }
};

// Writes line(i, s) for i in [0, n): chunks of lines formatted in parallel, written in order.
template <typename Line>
void put_lines(File& out, int64_t n, Line line) {
    constexpr int64_t kChunk = 1 << 15;
    const int64_t nch = (n + kChunk - 1) / kChunk;
    const int nt = std::max(1, omp_get_max_threads());
    std::vector<std::string> buf((size_t)nt);
    for (int64_t c0 = 0; c0 < nch && out.err.empty(); c0 += nt) {
        const int64_t c1 = std::min<int64_t>(nch, c0 + nt);
#pragma omp parallel for schedule(static, 1)
        for (int64_t c = c0; c < c1; ++c) {
            std::string& s = buf[(size_t)(c - c0)];
            s.clear();
            const int64_t e = std::min(n, (c + 1) * kChunk);
            for (int64_t i = c * kChunk; i < e; ++i) line(i, s);
        }
        for (int64_t c = c0; c < c1; ++c) out.put(buf[(size_t)(c - c0)]);
    }
}

void put_xyz(std::string& s, const double* p) {
    put_num(s, p[0]);
    s += ' ';
    put_num(s, p[1]);
    s += ' ';
    put_num(s, p[2]);
    s += '\n';
}

void vtu_head(File& out, int64_t npts, int64_t ncells, int64_t n, const double* pos) {
    out.put("<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n<UnstructuredGrid>\n");
    std::string s = "<Piece NumberOfPoints=\"";
    put_int(s, npts);
    s += "\" NumberOfCells=\"";
    put_int(s, ncells);
    s += "\">\n<Points>\n<DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    out.put(s);
    put_lines(out, n, [&](int64_t i, std::string& t) { put_xyz(t, pos + 3 * i); });
    out.put("</DataArray>\n</Points>\n");
}

void vtu_tail(File& out, int64_t n, const double* values, int ncomp) {
    out.put(ncomp == 3 ? "<PointData Scalars=\"value\">\n<DataArray type=\"Float64\" Name=\"value\" NumberOfComponents=\"3\" format=\"ascii\">\n"
                       : "<PointData Scalars=\"value\">\n<DataArray type=\"Float64\" Name=\"value\" format=\"ascii\">\n");
    if (values) {
        if (ncomp == 3)
            put_lines(out, n, [&](int64_t i, std::string& t) { put_xyz(t, values + 3 * i); });
        else
            put_lines(out, n, [&](int64_t i, std::string& t) {
                put_num(t, values[i]);
                t += '\n';
            });
    }
    out.put("</DataArray>\n</PointData>\n<CellData>\n</CellData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n");
}

std::string check(int64_t n, const double* pos, int ncomp) {
    if (n < 0 || (n > 0 && !pos)) return "invalid vertex array";
    if (ncomp != 1 && ncomp != 3) return "ncomp must be 1 or 3";
    return "";
}

}  // namespace

std::string write_vtu_tets(const char* path, int64_t n, const double* pos, int64_t ntet, const int32_t* tets, const double* values,
                           int ncomp) {
    std::string e = check(n, pos, ncomp);
    if (!e.empty()) return e;
    if (ntet < 0 || (ntet > 0 && !tets)) return "invalid tetrahedron array";
    File out(path);
    if (!out.err.empty()) return out.err;
    vtu_head(out, n, ntet, n, pos);
    out.put("<Cells>\n<DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n");
    put_lines(out, ntet, [&](int64_t t, std::string& s) {
        const int32_t* v = tets + 4 * t;
        for (int q = 0; q < 4; ++q) {
            put_int(s, v[q]);
            s += q < 3 ? ' ' : '\n';
        }
    });
    out.put("</DataArray>\n<DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n");
    put_lines(out, ntet, [&](int64_t t, std::string& s) {
        put_int(s, 4 * (t + 1));
        s += '\n';
    });
    out.put("</DataArray>\n<DataArray type=\"Int32\" Name=\"types\" format=\"ascii\">\n");
    put_lines(out, ntet, [&](int64_t, std::string& s) { s += "10\n"; });
    out.put("</DataArray>\n</Cells>\n");
    vtu_tail(out, n, values, ncomp);
    return out.close();
}

std::string write_vtu_points(const char* path, int64_t n, const double* pos, const double* values, int ncomp) {
    std::string e = check(n, pos, ncomp);
    if (!e.empty()) return e;
    File out(path);
    if (!out.err.empty()) return out.err;
    vtu_head(out, n, n, n, pos);
    out.put("<Cells>\n<DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n");
    put_lines(out, n, [&](int64_t i, std::string& s) {
        put_int(s, i);
        s += '\n';
    });
    out.put("</DataArray>\n<DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n");
    put_lines(out, n, [&](int64_t i, std::string& s) {
        put_int(s, i + 1);
        s += '\n';
    });
    out.put("</DataArray>\n<DataArray type=\"Int32\" Name=\"types\" format=\"ascii\">\n");
    put_lines(out, n, [&](int64_t, std::string& s) { s += "1\n"; });
    out.put("</DataArray>\n</Cells>\n");
    vtu_tail(out, n, values, ncomp);
    return out.close();
}

std::string write_csv(const char* path, int64_t n, const double* pos, const double* values, int ncomp) {
    std::string e = check(n, pos, ncomp);
    if (!e.empty()) return e;
    if (n > 0 && !values) return "values are NULL";
    File out(path);
    if (!out.err.empty()) return out.err;
    out.put(ncomp == 3 ? "x,y,z,value_x,value_y,value_z\n" : "x,y,z,value\n");
    put_lines(out, n, [&](int64_t i, std::string& s) {
        const double* p = pos + 3 * i;
        for (int q = 0; q < 3; ++q) {
            put_num(s, p[q]);
            s += ',';
        }
        for (int q = 0; q < ncomp; ++q) {
            put_num(s, values[ncomp * i + q]);
            s += q + 1 < ncomp ? ',' : '\n';
        }
    });
    return out.close();
}

}  // namespace vfv
