// Parallel cell-CSV reader/writer of include/b200ode_io.h.
//
// Reading: the whole file is read once, line starts are found, and the data
// lines are split into `threads` contiguous ranges parsed concurrently with
// std::from_chars into the structure-of-arrays buffers.  Writing: each thread
// formats a contiguous range of cells with std::to_chars (shortest form that
// parses back to the same double) into its own buffer; the buffers are written
// in order.
#include <algorithm>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "b200ode_io.h"

namespace {

thread_local std::string g_io_error;

int io_fail(const std::string& msg) {
    g_io_error = msg;
    return -1;
}

bool read_file(const char* path, std::string* out) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long len = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out->resize(len > 0 ? (size_t)len : 0);
    const size_t got = len > 0 ? std::fread(&(*out)[0], 1, (size_t)len, f) : 0;
    std::fclose(f);
    return got == out->size();
}

struct Header {
    int nsp = 0, ncols = 0;
    bool enthalpy = false, temperature = false, coords = false;
};

Header parse_header(const char* b, const char* e) {
    Header h;
    const char* p = b;
    while (p <= e) {
        const char* q = std::find(p, e, ',');
        const std::string col(p, q);
        ++h.ncols;
        if (col.find("CO") != std::string::npos) ++h.nsp;
        if (col.find("ENTHA") != std::string::npos) h.enthalpy = true;
        if (col.find("TEMPE") != std::string::npos) h.temperature = true;
        if (col.find("Points") != std::string::npos) h.coords = true;
        if (q == e) break;
        p = q + 1;
    }
    return h;
}

// Start offsets of the non-empty lines after the header, and the header's end.
void line_starts(const std::string& s, size_t* header_end, std::vector<size_t>* starts) {
    size_t p = s.find('\n');
    *header_end = (p == std::string::npos) ? s.size() : p;
    starts->clear();
    while (p != std::string::npos && p + 1 < s.size()) {
        const size_t b = p + 1;
        p = s.find('\n', b);
        const size_t e = (p == std::string::npos) ? s.size() : p;
        size_t k = b;
        while (k < e && (s[k] == '\r' || s[k] == ' ')) ++k;
        if (k < e) starts->push_back(b);
    }
}

int hw_threads(int t) {
    if (t > 0) return t;
    const unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}

const char* skip_sp(const char* p, const char* e) {
    while (p < e && (*p == ' ' || *p == '\t')) ++p;
    return p;
}

}  // namespace

extern "C" {

const char* b200ode_io_last_error(void) { return g_io_error.c_str(); }

int b200ode_csv_inspect(const char* path, b200ode_csv_info* info) {
    if (!path || !info) return io_fail("null argument");
    std::string s;
    if (!read_file(path, &s)) return io_fail(std::string("cannot read ") + path);
    size_t hend;
    std::vector<size_t> starts;
    line_starts(s, &hend, &starts);
    const char* b = s.data();
    const char* e = b + hend;
    while (e > b && (e[-1] == '\r' || e[-1] == ' ')) --e;
    const Header h = parse_header(b, e);
    if (!h.temperature) return io_fail(std::string(path) + ": no TEMPE column (the temperature is required)");
    info->n_cells = (int64_t)starts.size();
    info->n_species = h.nsp;
    info->has_enthalpy = h.enthalpy;
    info->has_coordinates = h.coords;
    return 0;
}

int b200ode_csv_read(const char* path, int32_t threads, double* T, double* Y, double* H, double* XYZ) {
    if (!path || !T || !Y) return io_fail("null argument");
    std::string s;
    if (!read_file(path, &s)) return io_fail(std::string("cannot read ") + path);
    size_t hend;
    std::vector<size_t> starts;
    line_starts(s, &hend, &starts);
    const char* e0 = s.data() + hend;
    while (e0 > s.data() && (e0[-1] == '\r' || e0[-1] == ' ')) --e0;
    const Header h = parse_header(s.data(), e0);
    if (!h.temperature) return io_fail(std::string(path) + ": no TEMPE column (the temperature is required)");
    const int64_t n = (int64_t)starts.size();
    const int nsp = h.nsp;
    const int nvals = nsp + (h.enthalpy ? 1 : 0) + 1 + (h.coords ? 3 : 0);
    const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(hw_threads(threads), n));
    std::vector<std::string> errors(nt);
    std::vector<std::thread> pool;
    auto work = [&](int t) {
        const int64_t c0 = n * t / nt, c1 = n * (t + 1) / nt;
        std::vector<double> v(nvals);
        for (int64_t c = c0; c < c1; ++c) {
            const char* p = s.data() + starts[c];
            const char* e = s.data() + ((c + 1 < n) ? starts[c + 1] : s.size());
            int got = 0;
            while (got < nvals) {
                p = skip_sp(p, e);
                double x = 0.0;
                const auto r = std::from_chars(p, e, x);
                if (r.ec != std::errc()) {
                    errors[t] = std::string(path) + ": line " + std::to_string(c + 2) + ", value " +
                                std::to_string(got + 1) + ": not a number";
                    return;
                }
                v[got++] = x;
                p = skip_sp(r.ptr, e);
                if (got < nvals) {
                    if (p >= e || *p != ',') {
                        errors[t] = std::string(path) + ": line " + std::to_string(c + 2) + ": " +
                                    std::to_string(got) + " values, expected " + std::to_string(nvals);
                        return;
                    }
                    ++p;
                }
            }
            int k = 0;
            for (int sp = 0; sp < nsp; ++sp) Y[(int64_t)sp * n + c] = v[k++];
            if (h.enthalpy) {
                if (H) H[c] = v[k];
                ++k;
            }
            T[c] = v[k++];
            if (h.coords && XYZ)
                for (int d = 0; d < 3; ++d) XYZ[(int64_t)d * n + c] = v[k + d];
        }
    };
    for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    for (const auto& m : errors)
        if (!m.empty()) return io_fail(m);
    return 0;
}

int b200ode_csv_write(const char* path, int64_t n, int32_t nsp, const double* T, const double* Y,
                      const double* H, const double* XYZ, int32_t threads) {
    if (!path || (n > 0 && (!T || !Y)) || n < 0 || nsp < 1) return io_fail("bad argument");
    std::string head;
    for (int k = 0; k < nsp; ++k) head += "CO" + std::to_string(k) + ",";
    if (H) head += "ENTHA,";
    head += "TEMPE";
    if (XYZ) head += ",Points:0,Points:1,Points:2";
    head += "\n";
    const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(hw_threads(threads), std::max<int64_t>(n, 1)));
    std::vector<std::string> out(nt);
    auto work = [&](int t) {
        const int64_t c0 = n * t / nt, c1 = n * (t + 1) / nt;
        std::string& o = out[t];
        o.reserve((size_t)(c1 - c0) * (size_t)(nsp + 5) * 24);
        char buf[64];
        auto put = [&](double x, char sep) {
            const auto r = std::to_chars(buf, buf + sizeof(buf), x);
            o.append(buf, r.ptr);
            o.push_back(sep);
        };
        for (int64_t c = c0; c < c1; ++c) {
            for (int k = 0; k < nsp; ++k) put(Y[(int64_t)k * n + c], ',');
            if (H) put(H[c], ',');
            put(T[c], XYZ ? ',' : '\n');
            if (XYZ)
                for (int d = 0; d < 3; ++d) put(XYZ[(int64_t)d * n + c], d < 2 ? ',' : '\n');
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    FILE* f = std::fopen(path, "wb");
    if (!f) return io_fail(std::string("cannot write ") + path);
    bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
    for (const auto& o : out) ok = ok && std::fwrite(o.data(), 1, o.size(), f) == o.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? 0 : io_fail(std::string("write failed: ") + path);
}

}  // extern "C"
