// ingest.cpp - fast `.jacob` input (JacobianIO.cpp:32-63) and its binary form.
//
// The text format is whitespace-separated:
//   lambda numCams camParams numPoints numObs
//   fix0 fix1 fix2
//   nrows ncols nnz
//   rowptr[nrows+1] cols[nnz] values[nnz]
// ('#' starts a comment to the end of the line, as in the documented template).
// The reference reads it with `ifstream >>` one number at a time; at 2000
// cameras / 500k points that is ~84M numbers. Here the file is read once, cut
// into per-thread chunks at whitespace, each chunk's tokens are counted, a
// prefix sum gives every chunk its first token index, and every thread parses
// its tokens straight into place (std::from_chars: correctly rounded, like
// strtod).
//
// Binary form (no counterpart in the reference): 64-byte header
//   "UNCJACB1" | f64 lambda | i32 numCams camParams numPoints numObs fix0 fix1
//   fix2 nrows ncols | i64 nnz | zero padding
// followed by i32 rowptr[nrows+1], i32 cols[nnz], f64 values[nnz] (little
// endian, the in-memory layout of the arrays).
#include <algorithm>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "uncte.h"

namespace unc {
extern thread_local std::string g_last_error;  // unc_last_error()
}

namespace {

constexpr char kMagic[8] = {'U', 'N', 'C', 'J', 'A', 'C', 'B', '1'};
constexpr size_t kBinHeader = 64;

int fail(const std::string& m) {
    unc::g_last_error = m;
    return UNC_ERR_INVALID_ARG;
}

bool read_file(const char* path, std::vector<char>& buf, size_t limit = 0) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    long long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (n < 0) {
        std::fclose(f);
        return false;
    }
    if (limit && (size_t)n > limit) n = (long long)limit;
    buf.resize((size_t)n + 1);
    size_t got = n ? std::fread(buf.data(), 1, (size_t)n, f) : 0;
    std::fclose(f);
    buf[got] = '\0';
    buf.resize(got + 1);
    return true;
}

inline bool is_ws(char c) { return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\f' || c == '\v'; }

// blank out comments so that they read as whitespace
void strip_comments(char* p, size_t n) {
    for (size_t i = 0; i < n; ++i)
        if (p[i] == '#')
            while (i < n && p[i] != '\n') p[i++] = ' ';
}

bool parse_header_tokens(const char* p, const char* end, unc_jacob_header* h, const char** after) {
    double vals[11];
    for (int t = 0; t < 11; ++t) {
        while (p < end && is_ws(*p)) ++p;
        if (p >= end) return false;
        auto r = std::from_chars(p, end, vals[t]);
        if (r.ec != std::errc()) return false;
        p = r.ptr;
    }
    h->lambda = vals[0];
    h->num_cams = (int)vals[1];
    h->cam_params = (int)vals[2];
    h->num_points = (int)vals[3];
    h->num_obs = (int)vals[4];
    for (int i = 0; i < 3; ++i) h->pts2fix[i] = (int)vals[5 + i];
    h->num_rows = (int)vals[8];
    h->num_cols = (int)vals[9];
    h->nnz = (long long)vals[10];
    h->binary = 0;
    if (after) *after = p;
    return true;
}

bool header_sane(const unc_jacob_header* h) {
    return h->num_rows >= 0 && h->num_cols >= 0 && h->nnz >= 0 && h->num_cams >= 0 && h->num_points >= 0;
}

}  // namespace

extern "C" {

int unc_jacob_read_header(const char* path, unc_jacob_header* h) {
    unc::g_last_error.clear();
    if (!path || !h) return fail("unc_jacob_read_header: null argument");
    std::vector<char> buf;
    if (!read_file(path, buf, 1 << 16)) return fail(std::string("cannot open ") + path);
    const size_t n = buf.size() - 1;
    if (n >= kBinHeader && std::memcmp(buf.data(), kMagic, 8) == 0) {
        const char* p = buf.data() + 8;
        std::memcpy(&h->lambda, p, 8);
        int32_t iv[9];
        std::memcpy(iv, p + 8, sizeof(iv));
        h->num_cams = iv[0];
        h->cam_params = iv[1];
        h->num_points = iv[2];
        h->num_obs = iv[3];
        for (int i = 0; i < 3; ++i) h->pts2fix[i] = iv[4 + i];
        h->num_rows = iv[7];
        h->num_cols = iv[8];
        int64_t nnz;
        std::memcpy(&nnz, p + 8 + sizeof(iv), 8);
        h->nnz = nnz;
        h->binary = 1;
        return header_sane(h) ? UNC_OK : fail("corrupt binary .jacob header");
    }
    strip_comments(buf.data(), n);
    if (!parse_header_tokens(buf.data(), buf.data() + n, h, nullptr) || !header_sane(h))
        return fail(std::string("bad .jacob header in ") + path);
    return UNC_OK;
}

int unc_jacob_read(const char* path, const unc_jacob_header* h, int* rows, int* cols, double* values) {
    unc::g_last_error.clear();
    if (!path || !h || !rows || (h->nnz && (!cols || !values))) return fail("unc_jacob_read: null argument");
    std::vector<char> buf;
    if (!read_file(path, buf)) return fail(std::string("cannot open ") + path);
    const size_t n = buf.size() - 1;
    const size_t nr = (size_t)h->num_rows + 1, nz = (size_t)h->nnz;
    if (h->binary) {
        const size_t need = kBinHeader + 4 * nr + 4 * nz + 8 * nz;
        if (n < need || std::memcmp(buf.data(), kMagic, 8) != 0) return fail("binary .jacob shorter than its header says");
        const char* p = buf.data() + kBinHeader;
        std::memcpy(rows, p, 4 * nr);
        std::memcpy(cols, p + 4 * nr, 4 * nz);
        std::memcpy(values, p + 4 * nr + 4 * nz, 8 * nz);
        return UNC_OK;
    }
    char* base = buf.data();
    strip_comments(base, n);
    unc_jacob_header hh;
    const char* body = nullptr;
    if (!parse_header_tokens(base, base + n, &hh, &body)) return fail("bad .jacob header");
    if (hh.num_rows != h->num_rows || hh.nnz != h->nnz) return fail("header does not match the file");
    const size_t start = (size_t)(body - base);
    const size_t total = nr + 2 * nz;
    // chunks cut at whitespace
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    if (n - start < (size_t)1 << 20) nt = 1;
    std::vector<size_t> cut(nt + 1);
    cut[0] = start;
    cut[nt] = n;
    for (unsigned t = 1; t < nt; ++t) {
        size_t c = start + (n - start) * t / nt;
        while (c < n && !is_ws(base[c])) ++c;
        cut[t] = std::max(c, cut[t - 1]);
    }
    std::vector<size_t> count(nt, 0);
    auto count_chunk = [&](unsigned t) {
        size_t k = 0;
        bool in = false;
        for (size_t i = cut[t]; i < cut[t + 1]; ++i) {
            const bool w = is_ws(base[i]);
            if (!w && !in) ++k;
            in = !w;
        }
        count[t] = k;
    };
    std::vector<int> bad(nt, 0);
    std::vector<size_t> first(nt + 1, 0);
    auto parse_chunk = [&](unsigned t) {
        size_t tok = first[t];
        const char* p = base + cut[t];
        const char* e = base + cut[t + 1];
        while (true) {
            while (p < e && is_ws(*p)) ++p;
            if (p >= e) break;
            if (tok < nr) {
                auto r = std::from_chars(p, e, rows[tok]);
                if (r.ec != std::errc()) { bad[t] = 1; return; }
                p = r.ptr;
            } else if (tok < nr + nz) {
                auto r = std::from_chars(p, e, cols[tok - nr]);
                if (r.ec != std::errc()) { bad[t] = 1; return; }
                p = r.ptr;
            } else if (tok < total) {
                auto r = std::from_chars(p, e, values[tok - nr - nz]);
                if (r.ec != std::errc()) { bad[t] = 1; return; }
                p = r.ptr;
            } else {
                bad[t] = 1;
                return;
            }
            ++tok;
        }
    };
    auto run = [&](auto&& fn) {
        std::vector<std::thread> th;
        for (unsigned t = 1; t < nt; ++t) th.emplace_back(fn, t);
        fn(0u);
        for (auto& x : th) x.join();
    };
    run(count_chunk);
    for (unsigned t = 0; t < nt; ++t) first[t + 1] = first[t] + count[t];
    if (first[nt] != total)
        return fail("the file holds " + std::to_string(first[nt]) + " numbers after the header, expected " +
                    std::to_string(total));
    run(parse_chunk);
    for (unsigned t = 0; t < nt; ++t)
        if (bad[t]) return fail("malformed number in the .jacob body");
    return UNC_OK;
}

int unc_jacob_write_binary(const char* path, const unc_jacob_header* h, const int* rows, const int* cols,
                           const double* values) {
    unc::g_last_error.clear();
    if (!path || !h || !rows || (h->nnz && (!cols || !values))) return fail("unc_jacob_write_binary: null argument");
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(std::string("cannot create ") + path);
    char hdr[kBinHeader] = {0};
    std::memcpy(hdr, kMagic, 8);
    std::memcpy(hdr + 8, &h->lambda, 8);
    const int32_t iv[9] = {h->num_cams, h->cam_params, h->num_points, h->num_obs, h->pts2fix[0],
                           h->pts2fix[1], h->pts2fix[2], h->num_rows, h->num_cols};
    std::memcpy(hdr + 16, iv, sizeof(iv));
    const int64_t nnz = h->nnz;
    std::memcpy(hdr + 16 + sizeof(iv), &nnz, 8);
    const size_t nr = (size_t)h->num_rows + 1, nz = (size_t)h->nnz;
    bool ok = std::fwrite(hdr, 1, kBinHeader, f) == kBinHeader && std::fwrite(rows, 4, nr, f) == nr &&
              (nz == 0 || (std::fwrite(cols, 4, nz, f) == nz && std::fwrite(values, 8, nz, f) == nz));
    ok = (std::fclose(f) == 0) && ok;
    return ok ? UNC_OK : fail(std::string("write failed: ") + path);
}

}  // extern "C"
